// Column physics of the primitive-equation wet model for one column: large-scale
// condensation then the simplified Betts-Miller convection on the same state, tendencies
// added (SpeedyWeather/src/models/primitive_wet.jl:123-136).
//
//  * ImplicitCondensation: SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178
//  * BettsMillerConvection, pseudo_adiabat!: SpeedyWeather/src/parameterizations/convection.jl:33-253
//  * EarthAtmosphere constants: SpeedyWeather/src/dynamics/atmosphere.jl:14-73
//  * sigma coordinates with equispaced half levels: SpeedyWeather/src/dynamics/vertical_coordinates.jl:80-86
//  * geopotential from virtual temperature, flat orography: SpeedyWeather/src/dynamics/geopotential.jl:36-60
//
// Shared by the plain column kernel (column_physics.cu) and the fused emulator kernel
// (mlp.cu), which calls it for the columns outside the emulator's range.
#pragma once

#include "sht_internal.h"

namespace sht {
namespace colphys {

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

// tendencies dT [K/s], dq [kg/kg/s] of one column (T, q on the NL layers, top first; ps [Pa])
__device__ __forceinline__ void column_tendencies(const float (&T)[NL], const float (&q)[NL], float ps, float dt,
                                                  const Levels& L, float (&dT)[NL], float (&dq)[NL]) {
#pragma unroll
    for (int k = 0; k < NL; ++k) dT[k] = dq[k] = 0.f;

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
}

}  // namespace colphys

// sigma levels and geopotential coefficients (FP64 on the host, rounded once)
colphys::Levels column_levels();

}  // namespace sht
