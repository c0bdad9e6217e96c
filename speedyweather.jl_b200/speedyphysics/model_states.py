"""Columns of the wet primitive-equation model's own states at T63, for training the
column emulator.

No dynamical core is built here, so the states are the reference's initial state of the
PrimitiveWetModel (SpeedyWeather/src/dynamics/initial_conditions.jl:23-30):

* ZonalWind (:405-455): vorticity and divergence of the Jablonowski & Williamson (2006)
  baroclinic-wave test, eqs. 3, 12 and 13 (zonal jet, Gaussian perturbation), at the
  sigma level of each layer;
* JablonowskiTemperature (:593-710): eqs. 4 and 6 (no stratospheric term, as the
  reference's default dT = 0), T >= Tmin = 200 K, moist lapse rate 5 K/km;
* PressureOnOrography (:771-808) on flat orography: ln p_s = ln p0;
* ConstantRelativeHumidity (:831-880): q = 0.7 q_sat(T, sigma p_s);

each state with seeded variations standing in for the evolution a dynamical core would
produce: the jet's amplitude and the perturbation's centre and strength drawn per state,
a RandomVorticity field (:79-168: amplitude x l^(power+1), power -3, l <= 20, m > 0), and
large-scale random fields added to temperature (2 K), log surface pressure (1 %) and
relative humidity (0.2, clamped to 0.05 .. 1.05).

Every field passes through this library's transforms on the octahedral grid with nlat 96
(T63, one more degree for the vector fields): the grid functions are analysed, the
velocities come from UV_from_vordiv and a synthesis with unscale_coslat, temperature,
pressure and the random fields are synthesised from spectral space, as the model's
step produces its grid columns (SpeedyWeather/src/time_stepping/transform.jl:117-191).
"""
from __future__ import annotations

import math

import numpy as np
import torch

import speedytransforms as st

NLAYERS = 8
RADIUS = 6.371e6
ROTATION = 7.29e-5
GRAVITY = 9.81
R_DRY = 1000 * 8.3145 / 28.9649
R_VAPOUR = 1000 * 8.3145 / 18.0153
LATENT_HEAT = 2501.0e3
T_REF, P_REF, LAPSE = 288.0, 1.0e5, 5.0e-3
ETA0 = 0.252


def sigma_full(nlayers: int = NLAYERS):
    """Full sigma levels of equispaced half levels (the column physics' levels)."""
    return (np.arange(nlayers) + 0.5) / nlayers


def saturation_humidity(T, p):
    """Clausius-Clapeyron over water, as the column physics (atmosphere.jl:138-157)."""
    e_sat = 610.78 * torch.exp(LATENT_HEAT / R_VAPOUR * (1 / 273.15 - 1 / T))
    return (R_DRY / R_VAPOUR) * e_sat / p


def jw_vorticity(lon, lat, eta, u0, lonc, latc, up, R):
    """Relative vorticity [1/s] of the zonal jet plus the perturbation (J&W 2006 eqs. 3, 12)."""
    phi = torch.deg2rad(lat)
    sphi, cphi = torch.sin(phi), torch.cos(phi)
    sc, cc = math.sin(math.radians(latc)), math.cos(math.radians(latc))
    cdl = torch.cos(torch.deg2rad(lon - lonc))
    X = torch.clamp(sc * sphi + cc * cphi * cdl, 0.0, 1.0)
    r = RADIUS * torch.acos(X)
    cv = math.cos((eta - ETA0) * math.pi / 2)
    zeta = -4 * u0 / RADIUS * cv * math.sqrt(cv) * sphi * cphi * (2 - 5 * sphi ** 2)
    s = torch.sqrt(torch.clamp(1 - X ** 2, min=1e-30))
    pert = up / RADIUS * torch.exp(-(r / R) ** 2) * (
        torch.tan(phi) - 2 * (RADIUS / R) ** 2 * torch.acos(X) * (sc * cphi - cc * sphi * cdl) / s)
    return zeta + pert


def jw_divergence(lon, lat, up, lonc, latc, R):
    """Divergence [1/s] of the perturbation (J&W 2006 eq. 13)."""
    phi = torch.deg2rad(lat)
    sphi, cphi = torch.sin(phi), torch.cos(phi)
    sc, cc = math.sin(math.radians(latc)), math.cos(math.radians(latc))
    dl = torch.deg2rad(lon - lonc)
    X = torch.clamp(sc * sphi + cc * cphi * torch.cos(dl), 0.0, 1.0)
    r = RADIUS * torch.acos(X)
    s = torch.sqrt(torch.clamp(1 - X ** 2, min=1e-30))
    return -2 * up * RADIUS / R ** 2 * torch.exp(-(r / R) ** 2) * torch.acos(X) / s * cc * torch.sin(dl)


def jw_temperature(lat, eta, u0):
    """Temperature [K] (J&W 2006 eqs. 4, 6) with the reference's default: no stratospheric term."""
    T_eta = max(T_REF * eta ** (R_DRY * LAPSE / GRAVITY), 200.0)
    ev = (eta - ETA0) * math.pi / 2
    cv = math.cos(ev)
    A1 = 0.75 * eta * math.pi * u0 / R_DRY * math.sin(ev) * math.sqrt(cv)
    A2 = 2 * u0 * cv * math.sqrt(cv)
    phi = torch.deg2rad(lat)
    sphi, cphi = torch.sin(phi), torch.cos(phi)
    return T_eta + A1 * ((-2 * sphi ** 6 * (cphi ** 2 + 1.0 / 3) + 10.0 / 63) * A2
                         + (1.6 * cphi ** 3 * (sphi ** 2 + 2.0 / 3) - math.pi / 4) * RADIUS * ROTATION)


class ModelStates:
    """The T63 transform and grid coordinates, and states(seed) -> columns."""

    def __init__(self, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.spec = st.Spectrum(65, 64)
        self.grid = st.OctahedralGaussianGrid(48)
        self.S = st.SpectralTransform(self.spec, self.grid, nlayers=NLAYERS, precision="fp32", device=self.device)
        g = self.grid
        lat = np.repeat(self.S.latd, g.nlons)
        lon = np.concatenate([360.0 * np.arange(n) / n for n in g.nlons])
        self.lat = torch.tensor(lat, dtype=torch.float64, device=self.device)
        self.lon = torch.tensor(lon, dtype=torch.float64, device=self.device)
        lidx = np.concatenate([np.arange(m, self.spec.lmax) for m in range(self.spec.mmax)])
        midx = np.concatenate([np.full(self.spec.lmax - m, m) for m in range(self.spec.mmax)])
        self.l = torch.tensor(lidx, dtype=torch.float64, device=self.device)
        self.m = torch.tensor(midx, device=self.device)
        self.ncol = g.npoints

    def _lta(self, c):
        return st.LowerTriangularArray(c.to(torch.complex64).contiguous(), self.spec)

    def _field(self, f):
        return st.Field(f.to(torch.float32).contiguous(), self.grid)

    def _random_field(self, gen, K, lmax=20, power=-1.5):
        """Grid fields of K layers synthesised from random coefficients ~ (l+1)^power, l <= lmax,
        normalised to unit standard deviation per layer."""
        n = self.spec.nlm
        re = torch.randn((K, n), generator=gen, device=self.device, dtype=torch.float64)
        im = torch.randn((K, n), generator=gen, device=self.device, dtype=torch.float64)
        amp = torch.where(self.l <= lmax, (self.l + 1) ** power, torch.zeros_like(self.l))
        c = torch.complex(re, torch.where(self.m == 0, torch.zeros_like(im), im)) * amp
        f = st.transform(self._lta(c), self.S).data.double()
        return f / f.std(dim=1, keepdim=True).clamp(min=1e-30)

    def state(self, seed: int):
        """(temp, humid, u, v [8, ncol], surface_pressure [ncol]) float32 of one seeded state."""
        gen = torch.Generator(device=self.device).manual_seed(int(seed))
        U = lambda: float(torch.rand(1, generator=gen, device=self.device))   # noqa: E731
        sig = sigma_full()
        u0 = 35.0 * (0.8 + 0.4 * U())
        lonc, latc = 360.0 * U(), (20.0 + 40.0 * U()) * (1 if U() < 0.5 else -1)
        up, R = 0.5 + 1.5 * U(), RADIUS / 10
        S, K = self.S, NLAYERS
        zeta = torch.stack([jw_vorticity(self.lon, self.lat, e, u0, lonc, latc, up, R) for e in sig])
        div = jw_divergence(self.lon, self.lat, up, lonc, latc, R).expand(K, -1)
        vor_c = st.transform(self._field(zeta), S).data.to(torch.complex128)
        div_c = st.transform(self._field(div), S).data.to(torch.complex128)
        # RandomVorticity (initial_conditions.jl:79-168): amplitude l^(power + 1) x U(-1, 1), l <= 20, m > 0
        amp = 1e-4 * (0.5 + U())
        rr = 2 * torch.rand((K, self.spec.nlm), generator=gen, device=self.device, dtype=torch.float64) - 1
        ri = 2 * torch.rand((K, self.spec.nlm), generator=gen, device=self.device, dtype=torch.float64) - 1
        mask = (self.m > 0) & (self.l <= 20)
        vor_c = vor_c + torch.where(mask, amp * self.l.clamp(min=1) ** -2.0, torch.zeros_like(self.l)) * torch.complex(
            rr, ri)
        Uc, Vc = st.UV_from_vordiv(self._lta(vor_c), self._lta(div_c), S, radius=RADIUS)
        u = st.transform(Uc, S, unscale_coslat=True).data
        v = st.transform(Vc, S, unscale_coslat=True).data
        temp = torch.stack([jw_temperature(self.lat, e, u0) for e in sig]) + 2.0 * self._random_field(gen, K)
        temp = st.transform(st.transform(self._field(temp), S), S).data.double()     # spectral, then grid
        lnps = math.log(P_REF) + 0.01 * self._random_field(gen, 1)[0]
        ps = torch.exp(st.transform(st.transform(self._field(lnps[None]), S), S).data.double()[0])
        rh = torch.clamp(0.7 + 0.2 * self._random_field(gen, K), 0.05, 1.05)
        q = rh * saturation_humidity(temp, torch.tensor(sig, device=self.device)[:, None] * ps[None, :])
        f32 = lambda a: a.to(torch.float32).contiguous()   # noqa: E731
        return f32(temp), f32(q), f32(u), f32(v), f32(ps)

    def columns(self, seeds):
        """The states of the given seeds side by side: [8, len(seeds) ncol] and [len(seeds) ncol]."""
        parts = [self.state(s) for s in seeds]
        return tuple(torch.cat([p[i] for p in parts], dim=-1).contiguous() for i in range(5))
