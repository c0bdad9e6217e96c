"""Column-physics oracle: large-scale condensation and simplified Betts-Miller convection.

TEST INFRASTRUCTURE ONLY: a numpy restatement of the reference's column
parameterizations, used as the checker of the CUDA column-physics kernel and as the
teacher and the reference of the MLP emulator's tests. Never imported by the product path.

Follows, per column (vectorised over columns; FP64 by default, FP32 with dtype=float32):
* ImplicitCondensation: SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178
* BettsMillerConvection and pseudo_adiabat!: SpeedyWeather/src/parameterizations/convection.jl:33-253
* saturation_humidity (Clausius-Clapeyron): SpeedyWeather/src/dynamics/atmosphere.jl:138-157
* EarthAtmosphere constants: SpeedyWeather/src/dynamics/atmosphere.jl:14-73; gravity
  SpeedyWeather/src/dynamics/planet.jl:6
* sigma coordinates (equispaced half levels, midpoints, thickness):
  SpeedyWeather/src/dynamics/vertical_coordinates.jl:44-86, 107-125
* geopotential on full levels from virtual temperature: SpeedyWeather/src/dynamics/geopotential.jl:36-60,113-131
  (flat orography)
* the two schemes run on the same state and add their tendencies
  (SpeedyWeather/src/models/primitive_wet.jl:123-136, tendencies accumulate).

Parity with the reference's own runs is unpinned (no Julia toolchain here); the
restatement is pinned by the invariants in tests/test_column_oracle.py.

The MLP emulator (no counterpart in the reference) has its forward and backward pass
restated here too (mlp_forward, mlp_backward): FP64 arithmetic with BF16 rounding at the
points where the CUDA kernels store BF16 (normalised inputs, weights, hidden activations,
output and hidden gradients), or exact FP64 (bf16=False), which finite differences pin.
"""
from __future__ import annotations

import numpy as np

# EarthAtmosphere defaults
MOL_MASS_DRY, MOL_MASS_VAPOR = 28.9649, 18.0153
CP = 1004.0
R_GAS = 8.3145
R_DRY = 1000 * R_GAS / MOL_MASS_DRY
R_VAPOR = 1000 * R_GAS / MOL_MASS_VAPOR
EPS = R_DRY / R_VAPOR                      # mol_ratio
MU_VIRT = (1 - EPS) / EPS
KAPPA = R_DRY / CP
RHO_WATER = 1000.0
LV, LF = 2501.0e3, 3.3e5
E0, T0 = 610.78, 273.15
GRAVITY = 9.81
# ImplicitCondensation defaults
RH_THRESHOLD, REEVAPORATION, FREEZING, MELTING, COND_TIME_SCALE = 0.95, 30.0, 263.0, 278.0, 3.0
# BettsMillerConvection defaults
CONV_TIME_SCALE, CONV_RH = 4 * 3600.0, 0.7
DT_T63 = 1200.0                            # time step at T63 [s]


def sigma_levels(nlayers: int = 8):
    half = np.linspace(0.0, 1.0, nlayers + 1)
    half[0] = 0.0
    return half, 0.5 * (half[1:] + half[:-1]), half[1:] - half[:-1]


def saturation_humidity(T, p):
    return EPS * E0 * np.exp(LV / R_VAPOR * (1.0 / T0 - 1.0 / T)) / p


def virtual_temperature(T, q):
    return T * (1 + MU_VIRT * q)


def geopotential(T, q, nlayers: int = 8, dtype=np.float64):
    """Phi [ncol, nlayers] on full levels, flat orography (geopotential.jl:113-131)."""
    half, full, _ = sigma_levels(nlayers)
    dhalf = np.zeros(nlayers, dtype=dtype)
    dhalf[1:] = R_DRY * np.log(full[1:] / half[1:nlayers])
    dfull = (R_DRY * np.log(half[1:] / full)).astype(dtype)
    Tv = virtual_temperature(T, q)
    phi = np.zeros_like(T)
    phi[:, -1] = Tv[:, -1] * dfull[-1]
    for k in range(nlayers - 2, -1, -1):
        phi[:, k] = phi[:, k + 1] + Tv[:, k + 1] * dhalf[k + 1] + Tv[:, k] * dfull[k]
    return phi


def condensation(T, q, ps, dt=DT_T63, dtype=np.float64):
    """Tendencies (dT/dt [K/s], dq/dt [kg/kg/s]) of ImplicitCondensation; T, q [ncol, nl]."""
    f = dtype
    T, q, ps = T.astype(f), q.astype(f), ps.astype(f)
    ncol, nl = T.shape
    _, full, dsig = sigma_levels(nl)
    dT = np.zeros_like(T)
    dq = np.zeros_like(T)
    rain = np.zeros(ncol, f)
    snow = np.zeros(ncol, f)
    g_rho = f(GRAVITY * RHO_WATER)
    lv_cp, lf_cp, cp_lf = f(LV / CP), f(LF / CP), f(CP / LF)
    for k in range(nl):
        pk = f(full[k]) * ps
        qsat = saturation_humidity(T[:, k], pk).astype(f)
        dq_cond = qsat * f(RH_THRESHOLD) - q[:, k]
        act = (dq_cond < 0) | (snow > 0) | (rain > 0)
        dp = f(dsig[k]) * ps
        dp_grho = dp / g_rho
        dp_dtgrho = dp_grho / f(dt)
        dtgrho_dp = 1 / dp_dtgrho
        dT_melt = np.maximum(T[:, k] - f(MELTING), 0)
        melt_max = cp_lf * dT_melt * dp_dtgrho
        melt = np.minimum(snow, melt_max)
        snow_a = snow - melt
        rain_a = rain + melt
        dT_l = -lf_cp * (melt * dtgrho_dp)
        r = f(REEVAPORATION) * np.maximum(qsat - q[:, k], 0)
        evap = np.minimum(r, 1) * rain_a
        rain_a = rain_a - evap
        dqk = np.minimum(0, dq_cond) + evap * dtgrho_dp
        Tn = T[:, k] + f(dt) * dT_l
        dqsat_dT = qsat * f(RH_THRESHOLD) * lv_cp / (f(R_VAPOR) * Tn * Tn)
        dqk = dqk / ((1 + lv_cp * dqsat_dT) * f(COND_TIME_SCALE) * f(dt))
        dTk = -lv_cp * dqk
        dq_rain = np.minimum(0, dqk)
        r_k = dp_grho * -dq_rain
        frozen = T[:, k] < f(FREEZING)
        s_k = np.where(frozen, r_k, 0)
        r_k = np.where(frozen, 0, r_k)
        rain_a = rain_a + r_k
        snow_a = snow_a + s_k
        dTk = dTk - (s_k > 0) * lf_cp * dq_rain
        dq[:, k] = np.where(act, dqk, 0)
        dT[:, k] = np.where(act, dTk, 0)
        rain = np.where(act, rain_a, rain)
        snow = np.where(act, snow_a, snow)
    return dT, dq


def convection(T, q, ps, dtype=np.float64):
    """Tendencies of BettsMillerConvection (qref formulation) with pseudo_adiabat!."""
    f = dtype
    T, q, ps = T.astype(f), q.astype(f), ps.astype(f)
    ncol, nl = T.shape
    half, full, dsig = sigma_levels(nl)
    phi = geopotential(T, q, nl, f)
    dT = np.zeros_like(T)
    dq = np.zeros_like(T)
    for c in range(ncol):
        Tc, qc, p = T[c], q[c], ps[c]
        Tref = np.full(nl, np.nan, f)
        Tp, qp = Tc[-1], qc[-1]
        Tref[-1] = Tp
        saturated, buoyant, k = False, True, nl - 1
        Tvp = virtual_temperature(Tp, qp)
        while buoyant and k > 0:
            k -= 1
            if not saturated:
                Tdry = Tp * f((full[k] / full[k + 1]) ** KAPPA)
                qs = f(saturation_humidity(Tdry, f(full[k]) * p))
                saturated = qp >= qs
            if saturated:
                A = qp * f(LV) / ((1 - qp) ** 2 * f(R_DRY))
                B = qp * f(LV) ** 2 / ((1 - qp) ** 2 * f(CP) * f(R_VAPOR))
                gam = (1 + A / Tvp) / (1 + B / (Tp * Tp))
                dphi = phi[c, k] - phi[c, k + 1]
                Tp = Tp - dphi / f(CP) * gam
                qp = f(saturation_humidity(Tp, f(full[k]) * p))
            else:
                Tp = Tdry
            Tref[k] = Tp
            Tvp = virtual_temperature(Tp, qp)
            buoyant = Tvp > virtual_temperature(Tc[k], qc[k])
        if not buoyant:
            Tref[k] = np.nan
        lzb = k + (0 if buoyant else 1)                  # 0-based first level of the profile
        lev = slice(lzb, nl)
        qref = np.zeros(nl, f)
        qref[lev] = saturation_humidity(Tref[lev], p * full[lev]).astype(f) * f(CONV_RH)
        Pq = np.sum((qc[lev] - qref[lev]) * dsig[lev].astype(f))
        PT = -np.sum((Tc[lev] - Tref[lev]) * dsig[lev].astype(f))
        deep = Pq > 0 and PT > 0
        shallow = Pq <= 0 and PT > 0
        if not (deep or shallow):
            continue
        dsig_lzb = f(half[nl] - half[lzb])
        if deep:
            Tref[lev] -= (PT - Pq * f(LV) / f(CP)) / dsig_lzb
        else:
            Qref = -np.sum(qref[lev] * dsig[lev].astype(f))
            qref[lev] *= 1 - Pq / Qref
            Tref[lev] -= PT / dsig_lzb
        tau_inv = f(1.0 / CONV_TIME_SCALE)
        dT[c, lev] -= (Tc[lev] - Tref[lev]) * tau_inv
        dq[c, lev] -= (qc[lev] - qref[lev]) * tau_inv
    return dT, dq


def column_tendencies(T, q, ps, dt=DT_T63, dtype=np.float64):
    """Condensation + convection tendencies, each [ncol, nlayers]."""
    a = condensation(T, q, ps, dt, dtype)
    b = convection(T, q, ps, dtype)
    return a[0] + b[0], a[1] + b[1]


def synthetic_columns(ncol: int, seed: int = 0, nlayers: int = 8):
    """Seeded columns standing in for model-generated states (no dynamical core here):
    latitude-dependent surface temperature with a tropospheric lapse rate, relative
    humidity from 0.2 to 1.05 decreasing upward, a zonal jet with noise, log surface
    pressure near 1e5 Pa. Returns T, q, u, v [ncol, nlayers] and ps [ncol], float32."""
    rng = np.random.default_rng(seed)
    _, full, _ = sigma_levels(nlayers)
    lat = np.arcsin(rng.uniform(-1, 1, ncol))
    ps = 1e5 * np.exp(rng.normal(0, 0.02, ncol))
    Ts = 302 - 45 * np.sin(lat) ** 2 + rng.normal(0, 3, ncol)
    T = Ts[:, None] * full[None, :] ** (R_DRY * 0.0065 / GRAVITY) + rng.normal(0, 1.5, (ncol, nlayers))
    T = np.maximum(T, 195.0 + rng.normal(0, 2, (ncol, nlayers)))
    rh_s = rng.uniform(0.5, 1.05, ncol)
    rh = rh_s[:, None] * (0.25 + 0.75 * full[None, :] ** 1.5) * rng.uniform(0.85, 1.15, (ncol, nlayers))
    q = np.clip(rh, 0.02, 1.08) * saturation_humidity(T, ps[:, None] * full[None, :])
    u = 30 * np.sin(2 * lat)[:, None] * (1.2 - full[None, :]) + rng.normal(0, 5, (ncol, nlayers))
    v = rng.normal(0, 4, (ncol, nlayers))
    return (T.astype(np.float32), q.astype(np.float32), u.astype(np.float32), v.astype(np.float32),
            ps.astype(np.float32))


# ---- MLP emulator: 33 -> 256 -> 256 -> 256 (GELU) -> 16 ----------------------------
def bf16_round(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    """GELU in its tanh form (Hendrycks & Gimpel 2016), as the emulator's kernels."""
    u = np.sqrt(2.0 / np.pi) * (x + 0.044715 * x ** 3)
    return 0.5 * x * (1 + np.tanh(u))


def gelu_grad(x):
    u = np.sqrt(2.0 / np.pi) * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    du = np.sqrt(2.0 / np.pi) * (1 + 3 * 0.044715 * x ** 2)
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * du


def mlp_forward(params, xn, bf16=True):
    """params: [(w [out][in], b [out])] * 4 with in = 64 for the first layer (inputs
    padded with zeros); xn [B, 33] normalised inputs. Returns (Y, cache)."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    B = xn.shape[0]
    a = np.zeros((B, params[0][0].shape[1]))
    a[:, :xn.shape[1]] = xn
    a = r(a)
    acts, zs = [a], []
    for layer, (w, b) in enumerate(params):
        z = a @ r(w).T + np.asarray(b, np.float64)
        if layer == len(params) - 1:
            return z, (acts, zs)
        zs.append(z)
        a = r(gelu(z))
        acts.append(a)


def mlp_backward(params, xn, yn, bf16=True):
    """Loss = mean over B x 16 of (Y - yn)^2 and its gradients [(dW, db)] * 4."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    Y, (acts, zs) = mlp_forward(params, xn, bf16)
    d = Y - yn
    loss = float(np.mean(d * d))
    dz = r(2 * d / d.size)
    grads = [None] * len(params)
    for layer in range(len(params) - 1, -1, -1):
        grads[layer] = (dz.T @ acts[layer], dz.sum(0))
        if layer > 0:
            dz = r((dz @ r(params[layer][0])) * gelu_grad(zs[layer - 1]))
    return loss, grads
