"""The spectral transforms of one time step of the primitive-equation wet model, in the
reference's order, on this library's calls: the sequence a dynamical core replays every
step, captured once as a CUDA graph (any sequence of these calls can be captured: none of
them allocates or synchronises).

Follows SpeedyWeather/src/time_stepping/transform.jl:117-191 (spectral to grid) and
SpeedyWeather/src/dynamics/tendencies.jl:161-214, 585-594 (pressure-gradient flux, the
batched grid-to-spectral transform of the tendencies, curl/divergence of the momentum
tendencies, flux divergences):

    ∇ ln p_s                                  (1 layer)  -> synthesis, unscale_coslat (2)
    UV_from_vordiv (U, V from vorticity, divergence)     (L)
    synthesis of vorticity, divergence, temperature, humidity, pressure   (4L + 1)
    synthesis of U, V, unscale_coslat                                      (2L)
    analysis of the grid tendencies u, v, T, p, uT, vT, KE, q, uq, vq      (9L + 1)
    curl and divergence of (u, v) tendencies, divergence of (uT, vT) and (uq, vq)
    fluxes, ∇² of the kinetic energy, accumulated into the spectral tendencies (L each)

The grid-space physics and dynamics between the two directions are outside this
library; their results (the grid tendencies) are the step's input here.

With fused=True (the default) the operators run as two sets of one kernel launch each
(``Operators``: the gradient with UV_from_vordiv, and the five operators on the analysed
tendencies), with the same results as the separate calls bit for bit: 7 library calls
per step instead of 11.
"""
from __future__ import annotations

import torch

from . import core as st


class DycoreStep:
    """Buffers and the call sequence of one step at truncation T (1-based size T + 1 with
    one more degree) on an octahedral Gaussian grid with nlat_half rings per hemisphere
    and L layers."""

    def __init__(self, T: int = 63, nlat_half: int = 48, L: int = 8, precision: str = "fp32", device=None, seed=0,
                 fused: bool = True):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.L = L
        self.fused = fused
        spec = st.Spectrum(T + 2, T + 1)
        grid = st.OctahedralGaussianGrid(nlat_half)
        self.S = st.SpectralTransform(spec, grid, nlayers=9 * L + 1, precision=precision, device=dev)
        g = torch.Generator(device="cpu").manual_seed(seed)
        l = torch.tensor(spec_degrees(spec), dtype=torch.float32)
        amp = (l + 1) ** -1.5

        def coeffs(K):
            c = torch.complex(torch.randn(K, spec.nlm, generator=g), torch.randn(K, spec.nlm, generator=g)) * amp
            return st.LowerTriangularArray(c.to(torch.complex64).to(dev), spec)

        z = lambda K: st.LowerTriangularArray.zeros(spec, K, device=dev)   # noqa: E731
        self.prog = coeffs(4 * L + 1)                      # vor, div, temp, humid, pres
        self.grid_prog = st.Field.zeros(grid, 4 * L + 1, device=dev)
        self.UV = z(2 * L)
        self.uv_grid = st.Field.zeros(grid, 2 * L, device=dev)
        self.dpres = z(2)
        self.dpres_grid = st.Field.zeros(grid, 2, device=dev)
        self.grid_tend = st.Field(torch.randn(9 * L + 1, grid.npoints, generator=g).to(dev), grid)
        self.spec_tend = z(9 * L + 1)
        self.tend = z(4 * L)                               # vor, div, temp, humid tendencies
        S, P, T = self.S, self.prog, self.spec_tend
        lta = self.lta
        self.ops_in = (st.Operators(S)
                       .gradient(lta(self.dpres, 0, 1), lta(self.dpres, 1, 2), lta(P, 4 * L, 4 * L + 1))
                       .UV_from_vordiv(lta(self.UV, 0, L), lta(self.UV, L, 2 * L), lta(P, 0, L), lta(P, L, 2 * L)))
        u, v = lta(T, 0, L), lta(T, L, 2 * L)
        vor_t, div_t = lta(self.tend, 0, L), lta(self.tend, L, 2 * L)
        temp_t, hum_t = lta(self.tend, 2 * L, 3 * L), lta(self.tend, 3 * L, 4 * L)
        self.ops_out = (st.Operators(S)
                        .curl(vor_t, u, v, add=True)
                        .divergence(div_t, u, v, add=True)
                        .divergence(temp_t, lta(T, 3 * L + 1, 4 * L + 1), lta(T, 4 * L + 1, 5 * L + 1), add=True,
                                    flipsign=True)
                        .divergence(hum_t, lta(T, 7 * L + 1, 8 * L + 1), lta(T, 8 * L + 1, 9 * L + 1), add=True,
                                    flipsign=True)
                        .laplace(div_t, lta(T, 5 * L + 1, 6 * L + 1), add=True, flipsign=True))

    def lta(self, x, a, b):
        return st.LowerTriangularArray(x.data[a:b], x.spectrum)

    def __call__(self):
        if self.fused:
            return self._fused()
        S, L = self.S, self.L
        P, T = self.prog, self.spec_tend
        self.tend.data.zero_()
        st.gradient_(self.lta(self.dpres, 0, 1), self.lta(self.dpres, 1, 2), self.lta(P, 4 * L, 4 * L + 1), S)
        st.transform_(self.dpres_grid, self.dpres, S, unscale_coslat=True)
        st.UV_from_vordiv_(self.lta(self.UV, 0, L), self.lta(self.UV, L, 2 * L), self.lta(P, 0, L),
                           self.lta(P, L, 2 * L), S)
        st.transform_(self.grid_prog, P, S)
        st.transform_(self.uv_grid, self.UV, S, unscale_coslat=True)
        st.transform_(T, self.grid_tend, S)
        u, v = self.lta(T, 0, L), self.lta(T, L, 2 * L)
        vor_t, div_t = self.lta(self.tend, 0, L), self.lta(self.tend, L, 2 * L)
        temp_t, hum_t = self.lta(self.tend, 2 * L, 3 * L), self.lta(self.tend, 3 * L, 4 * L)
        st.curl_(vor_t, u, v, S, add=True)
        st.divergence_(div_t, u, v, S, add=True)
        st.divergence_(temp_t, self.lta(T, 3 * L + 1, 4 * L + 1), self.lta(T, 4 * L + 1, 5 * L + 1), S,
                       add=True, flipsign=True)
        st.divergence_(hum_t, self.lta(T, 7 * L + 1, 8 * L + 1), self.lta(T, 8 * L + 1, 9 * L + 1), S,
                       add=True, flipsign=True)
        st.laplace_(div_t, self.lta(T, 5 * L + 1, 6 * L + 1), S, add=True, flipsign=True)

    def _fused(self):
        S = self.S
        self.tend.data.zero_()
        self.ops_in()
        st.transform_(self.dpres_grid, self.dpres, S, unscale_coslat=True)
        st.transform_(self.grid_prog, self.prog, S)
        st.transform_(self.uv_grid, self.UV, S, unscale_coslat=True)
        st.transform_(self.spec_tend, self.grid_tend, S)
        self.ops_out()

    def launches(self) -> int:
        """Library calls of one step (each one or more kernel launches)."""
        return 7 if self.fused else 11


def spec_degrees(spec):
    """0-based degree l of every packed coefficient (m-major)."""
    out = []
    for m in range(spec.mmax):
        out.extend(range(m, spec.lmax))
    return out
