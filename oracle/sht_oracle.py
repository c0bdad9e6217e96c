"""FP64 CPU oracle for the spherical harmonic transform (SHT) hot path.

TEST INFRASTRUCTURE ONLY. This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it. The product (``speedyweather.jl_b200``) never imports, links or
executes anything under ``oracle/``.

It restates, in plain numpy float64, what SpeedyTransforms computes:

* grid tables: ring lengths / offsets of the full and octahedral Gaussian grids
  (``RingGrids/src/grids/full_gaussian.jl:43-61``,
  ``RingGrids/src/grids/octahedral_gaussian.jl:50-116``), Gaussian latitudes and
  weights (``RingGrids/src/quadrature_weights.jl:11``), solid angles
  ``w_j 2pi / nlon_j`` (``RingGrids/src/quadrature_weights.jl:48-49``);
* the spectral layout (``LowerTriangularArrays/src/spectrum.jl:87-131``): packed
  lower triangle, order m outer, degree l inner;
* ``SpectralTransform`` precompute (``SpeedyTransforms/src/spectral_transform.jl:138-172``):
  Legendre shortcut, normalised associated Legendre polynomials;
* synthesis ``transform!(field, coeffs, S)``: Legendre
  (``SpeedyTransforms/src/legendre.jl:38-101``) then inverse real FFT per ring
  (``SpeedyTransforms/src/fourier.jl:215-250``);
* analysis ``transform!(coeffs, field, S)``: real FFT per ring
  (``SpeedyTransforms/src/fourier.jl:129-166``) then Legendre with quadrature
  (``SpeedyTransforms/src/legendre.jl:131-195``);
* the spectral operators (``SpeedyTransforms/src/spectral_gradients.jl``) with the
  factors of ``SpeedyTransforms/src/gradient_arrays.jl``.

Parity status. The reference is Julia and no Julia toolchain exists here, so
element-wise parity with the reference's own runs is unpinned. The oracle is
pinned instead against the reference's own known answers and invariant tests
(a_00 = 2 sqrt(pi) gives a grid of ones, ``spectral_transform.jl:158``;
single-harmonic round trips, ``SpeedyTransforms/test/spectral_transform.jl:71-102``;
band-limited round trips to 1e-13, ``:326-373``; operator identities,
``SpeedyTransforms/test/spectral_gradients.jl``), against closed-form Legendre
polynomials, and against numpy's Gauss-Legendre nodes.

Third-party arithmetic restated here: AssociatedLegendrePolynomials.jl v1.0.2
``lambdalm!`` (4pi-orthonormal "spherical harmonic" normalisation WITH the
Condon-Shortley phase (-1)^m, the package's documented convention; every
reference test is phase-invariant, so the phase is an assumption), computed by
the standard three-term recurrence; FastGaussQuadrature.jl v1.3.0
``gausslegendre`` (nodes ascending) restated by Newton iteration on P_n;
FFTW r2c / c2r (unnormalised; c2r ignores the imaginary parts of the DC and
Nyquist bins) restated by numpy's pocketfft.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

FULL_GAUSSIAN = 0
OCTAHEDRAL_GAUSSIAN = 1
GRID_NAMES = {FULL_GAUSSIAN: "FullGaussianGrid", OCTAHEDRAL_GAUSSIAN: "OctahedralGaussianGrid"}


# ----------------------------------------------------------------------------------------
# sizes (SpeedyTransforms/src/aliasing.jl:9-69)
# ----------------------------------------------------------------------------------------
def roundup_fft(n: int, small_primes=(2, 3, 5)) -> int:
    """Smallest even n' >= n with only ``small_primes`` as factors (aliasing.jl:41-59)."""
    n += n % 2
    while True:
        m = n
        for p in small_primes:
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 2


def get_nlat_half(truncation: int, dealiasing: float = 2.0) -> int:
    """aliasing.jl:9-15 (truncation is 1-based)."""
    return roundup_fft(math.ceil(((1 + dealiasing) * (truncation - 1) + 1) / 4))


def get_truncation(nlat_half: int, dealiasing: float = 2.0) -> int:
    """aliasing.jl:24-30."""
    return int(math.floor((4 * nlat_half - 1) / (dealiasing + 1))) + 1


# ----------------------------------------------------------------------------------------
# Gaussian quadrature (FastGaussQuadrature.gausslegendre, restated)
# ----------------------------------------------------------------------------------------
def gauss_legendre(n: int):
    """Nodes (ascending, -1..1) and weights of n-point Gauss-Legendre quadrature, FP64.

    Newton iteration on P_n from the Tricomi-like initial guess; the weights are
    2 / ((1 - x^2) P_n'(x)^2). Matches FastGaussQuadrature.gausslegendre to ~1e-15.
    """
    i = np.arange(1, n + 1, dtype=np.float64)
    x = np.cos(np.pi * (i - 0.25) / (n + 0.5))
    for _ in range(100):
        p0 = np.ones_like(x)
        p1 = x.copy()
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
        dp = n * (x * p1 - p0) / (x * x - 1.0)
        dx = p1 / dp
        x = x - dx
        if np.max(np.abs(dx)) < 1e-16:
            break
    p0 = np.ones_like(x)
    p1 = x.copy()
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    dp = n * (x * p1 - p0) / (x * x - 1.0)
    w = 2.0 / ((1.0 - x * x) * dp * dp)
    order = np.argsort(x)
    return x[order], w[order]


# ----------------------------------------------------------------------------------------
# grids (RingGrids)
# ----------------------------------------------------------------------------------------
@dataclass
class Grid:
    """Full or octahedral Gaussian ring grid, ring-major, rings north to south."""

    kind: int
    nlat_half: int
    nlat: int = field(init=False)
    nlons: np.ndarray = field(init=False)        # per ring, all nlat rings
    ring_start: np.ndarray = field(init=False)   # first point of each ring
    npoints: int = field(init=False)
    latd: np.ndarray = field(init=False)         # degrees, north to south
    weights: np.ndarray = field(init=False)      # Gaussian weights, pole to pole

    def __post_init__(self):
        nh = self.nlat_half
        self.nlat = 2 * nh
        if self.kind == FULL_GAUSSIAN:
            half = np.full(nh, 4 * nh, dtype=np.int64)                 # full_gaussian.jl:45
        elif self.kind == OCTAHEDRAL_GAUSSIAN:
            half = 16 + 4 * np.arange(1, nh + 1, dtype=np.int64)       # octahedral_gaussian.jl:64-70
        else:
            raise ValueError(f"unsupported grid kind {self.kind}")
        self.nlons = np.concatenate([half, half[::-1]])
        self.ring_start = np.concatenate([[0], np.cumsum(self.nlons)[:-1]]).astype(np.int64)
        self.npoints = int(self.nlons.sum())
        x, w = gauss_legendre(2 * nh)
        self.latd = np.degrees(np.arccos(x)) - 90.0                      # full_gaussian.jl:48-50
        self.weights = w                                                 # quadrature_weights.jl:11

    @property
    def nlons_half(self):
        return self.nlons[: self.nlat_half]

    @property
    def colat(self):
        return np.pi / 2 - np.radians(self.latd)                         # grid.jl:142-143

    @property
    def cos_colat(self):
        return np.cos(self.colat)

    @property
    def coslat(self):
        return np.cos(np.radians(self.latd))

    @property
    def solid_angles(self):
        return self.weights * (2 * np.pi / self.nlons)                  # quadrature_weights.jl:48-49

    def ring(self, j):
        s = int(self.ring_start[j])
        return slice(s, s + int(self.nlons[j]))

    def whichring(self):
        return np.repeat(np.arange(self.nlat), self.nlons)


# ----------------------------------------------------------------------------------------
# spectrum (LowerTriangularArrays/src/spectrum.jl)
# ----------------------------------------------------------------------------------------
@dataclass
class Spectrum:
    """Packed lower-triangular spectrum; lmax, mmax are 1-based sizes as in the reference."""

    lmax: int
    mmax: int

    def __post_init__(self):
        if self.lmax < self.mmax:
            raise ValueError("lmax must be >= mmax")
        self.nlm = self.lmax * self.mmax - self.mmax * (self.mmax - 1) // 2
        m_of = []
        l_of = []
        for m in range(self.mmax):
            for l in range(m, self.lmax):
                m_of.append(m)
                l_of.append(l)
        self.m_indices = np.array(m_of, dtype=np.int64)   # 0-based order of each lm
        self.l_indices = np.array(l_of, dtype=np.int64)   # 0-based degree of each lm

    def offset(self, m: int) -> int:
        """First packed index of order m (0-based)."""
        return m * self.lmax - m * (m - 1) // 2

    def lm(self, l: int, m: int) -> int:
        return self.offset(m) + (l - m)


# ----------------------------------------------------------------------------------------
# Legendre polynomials (AssociatedLegendrePolynomials.jl lambdalm!, restated)
# ----------------------------------------------------------------------------------------
def legendre_table(spectrum: Spectrum, x: np.ndarray, mmax_per_x=None) -> np.ndarray:
    """lambda_l^m(x) for all packed (l, m) and all x: array [nlm, len(x)], FP64.

    4pi-orthonormal with Condon-Shortley phase:
      lambda_00 = 1/sqrt(4pi)
      lambda_mm = -sqrt((2m+1)/(2m)) sqrt(1-x^2) lambda_{m-1,m-1}
      lambda_{m+1,m} = sqrt(2m+3) x lambda_mm
      lambda_lm = a_lm (x lambda_{l-1,m} - lambda_{l-2,m} / a_{l-1,m}),
      a_lm = sqrt((4l^2-1)/(l^2-m^2)).
    Orders above ``mmax_per_x[j]`` are left at zero (they are never used).
    """
    x = np.asarray(x, dtype=np.float64)
    nx = x.size
    lmax, mmax = spectrum.lmax, spectrum.mmax
    out = np.zeros((spectrum.nlm, nx))
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    pmm = np.full(nx, 1.0 / math.sqrt(4 * math.pi))
    mlim = np.full(nx, mmax - 1) if mmax_per_x is None else np.asarray(mmax_per_x)
    for m in range(mmax):
        if m > 0:
            pmm = -math.sqrt((2 * m + 1) / (2 * m)) * s * pmm
        use = m <= mlim
        o = spectrum.offset(m)
        out[o, :] = np.where(use, pmm, 0.0)
        if lmax - m >= 2:
            p1 = math.sqrt(2 * m + 3) * x * pmm
            out[o + 1, :] = np.where(use, p1, 0.0)
            p0 = pmm
            a_prev = math.sqrt((4 * (m + 1) ** 2 - 1) / ((m + 1) ** 2 - m * m))
            for l in range(m + 2, lmax):
                a = math.sqrt((4 * l * l - 1) / (l * l - m * m))
                p2 = a * (x * p1 - p0 / a_prev)
                out[o + l - m, :] = np.where(use, p2, 0.0)
                p0, p1, a_prev = p1, p2, a
    return out


# ----------------------------------------------------------------------------------------
# SpectralTransform (precompute) + transforms
# ----------------------------------------------------------------------------------------
SHORTCUTS = {
    "linear": lambda nlon, latd: nlon // 2,                               # legendre_shortcuts.jl:24
    "quadratic": lambda nlon, latd: nlon // 3,
    "cubic": lambda nlon, latd: nlon // 4,
    "linquadcoslat2": lambda nlon, latd: int(math.floor(nlon / (2 + math.cos(math.radians(latd)) ** 2))),
    "lincubcoslat": lambda nlon, latd: int(math.floor(nlon / (2 + 2 * math.cos(math.radians(latd))))),
}


class SpectralTransform:
    """FP64 restatement of SpeedyTransforms.SpectralTransform (spectral_transform.jl:118-302)."""

    def __init__(self, spectrum: Spectrum, grid: Grid, shortcut: str = "linear"):
        self.spectrum = spectrum
        self.grid = grid
        nh = grid.nlat_half
        nl = grid.nlons_half
        latd = grid.latd[:nh]
        mt = np.array([SHORTCUTS[shortcut](int(nl[j]), float(latd[j])) for j in range(nh)], dtype=np.int64)
        self.mmax_truncation = np.minimum(mt, spectrum.mmax - 1)          # spectral_transform.jl:154-155
        self.nfreq = nl // 2 + 1
        self.nfreq_max = int(grid.nlons.max()) // 2 + 1
        self.norm_sphere = 2 * math.sqrt(math.pi)
        self.lam = legendre_table(spectrum, grid.cos_colat[:nh], self.mmax_truncation)  # [nlm, nh]
        self.solid_angles = grid.solid_angles
        self.coslat = grid.coslat
        self.eigenvalues = -(np.arange(spectrum.lmax) * (np.arange(spectrum.lmax) + 1.0))
        ev_inv = np.zeros_like(self.eigenvalues)
        ev_inv[1:] = 1.0 / self.eigenvalues[1:]
        self.eigenvalues_inv = ev_inv

    # --- Legendre stages -------------------------------------------------------------
    def legendre_synthesis(self, coeffs, unscale_coslat=False):
        """g_north/g_south [nh, nfreq_max, K] (legendre.jl:38-101)."""
        sp, nh = self.spectrum, self.grid.nlat_half
        K = coeffs.shape[1]
        gN = np.zeros((nh, self.nfreq_max, K), dtype=np.complex128)
        gS = np.zeros_like(gN)
        mt = self.mmax_truncation
        for m in range(sp.mmax):
            rings = np.nonzero(mt >= m)[0]
            if rings.size == 0:
                continue
            o, L = sp.offset(m), sp.lmax - m
            lam = self.lam[o:o + L][:, rings]              # [L, nr]
            a = coeffs[o:o + L]                              # [L, K]
            even = lam[0::2].T @ a[0::2]                     # l - m even
            odd = lam[1::2].T @ a[1::2]
            gN[rings, m] = even + odd
            gS[rings, m] = even - odd
        if unscale_coslat:
            c = 1.0 / self.coslat[:nh]
            gN *= c[:, None, None]
            gS *= c[:, None, None]
        return gN, gS

    def legendre_analysis(self, fN, fS):
        """coeffs [nlm, K] from f_north/f_south (legendre.jl:131-195)."""
        sp, nh = self.spectrum, self.grid.nlat_half
        K = fN.shape[2]
        out = np.zeros((sp.nlm, K), dtype=np.complex128)
        mt = self.mmax_truncation
        w = self.solid_angles[:nh]
        for m in range(sp.mmax):
            rings = np.nonzero(mt >= m)[0]
            if rings.size == 0:
                continue
            o, L = sp.offset(m), sp.lmax - m
            lam = self.lam[o:o + L][:, rings]
            fn, fs = fN[rings, m], fS[rings, m]              # [nr, K]
            even = w[rings, None] * (fn + fs)
            odd = w[rings, None] * (fn - fs)
            out[o:o + L:2] = lam[0::2] @ even
            out[o + 1:o + L:2] = lam[1::2] @ odd
        return out

    # --- Fourier stages ---------------------------------------------------------------
    def fourier_synthesis(self, gN, gS):
        g = self.grid
        nh, K = g.nlat_half, gN.shape[2]
        field_ = np.zeros((g.npoints, K))
        for j in range(nh):
            n = int(g.nlons[j])
            nf = n // 2 + 1
            field_[g.ring(j)] = np.fft.irfft(gN[j, :nf], n=n, axis=0) * n
            field_[g.ring(g.nlat - 1 - j)] = np.fft.irfft(gS[j, :nf], n=n, axis=0) * n
        return field_

    def fourier_analysis(self, field_):
        g = self.grid
        nh, K = g.nlat_half, field_.shape[1]
        fN = np.zeros((nh, self.nfreq_max, K), dtype=np.complex128)
        fS = np.zeros_like(fN)
        for j in range(nh):
            n = int(g.nlons[j])
            nf = n // 2 + 1
            fN[j, :nf] = np.fft.rfft(field_[g.ring(j)], axis=0)
            fS[j, :nf] = np.fft.rfft(field_[g.ring(g.nlat - 1 - j)], axis=0)
        return fN, fS

    # --- full transforms ----------------------------------------------------------------
    def synthesize(self, coeffs, unscale_coslat=False):
        coeffs = np.asarray(coeffs, dtype=np.complex128)
        squeeze = coeffs.ndim == 1
        if squeeze:
            coeffs = coeffs[:, None]
        if coeffs.shape[0] != self.spectrum.nlm:
            raise ValueError("DimensionMismatch: coeffs do not match the spectrum")
        gN, gS = self.legendre_synthesis(coeffs, unscale_coslat)
        out = self.fourier_synthesis(gN, gS)
        return out[:, 0] if squeeze else out

    def analyze(self, field_):
        field_ = np.asarray(field_, dtype=np.float64)
        squeeze = field_.ndim == 1
        if squeeze:
            field_ = field_[:, None]
        if field_.shape[0] != self.grid.npoints:
            raise ValueError("DimensionMismatch: field does not match the grid")
        fN, fS = self.fourier_analysis(field_)
        out = self.legendre_analysis(fN, fS)
        return out[:, 0] if squeeze else out


    # --- adjoints (SpeedyTransforms/ext/SpeedyTransformsEnzymeExt.jl) ----------------
    def adjoint_scale(self):
        """rfft adjoint scale [nh, nfreq_max] (SpeedyTransformsEnzymeExt.jl:33-57): 1 for
        m = 0 and, for even n, the Nyquist frequency; 2 otherwise; 0 beyond the ring's."""
        nh = self.grid.nlat_half
        sc = np.zeros((nh, self.nfreq_max))
        for j in range(nh):
            n = int(self.grid.nlons[j])
            nf = n // 2 + 1
            s = np.full(nf, 2.0)
            s[0] = 1.0
            if n % 2 == 0:
                s[nf - 1] = 1.0
            sc[j, :nf] = s
        return sc

    def synthesize_adjoint(self, field_bar, unscale_coslat=False):
        """spec2grid_pullback! (SpeedyTransformsEnzymeExt.jl:263-289): forward FFT, times
        the adjoint scale (and 1/cos lat), divided by the solid angle that the forward
        Legendre applies, then the forward Legendre."""
        field_bar = np.asarray(field_bar, dtype=np.float64)
        squeeze = field_bar.ndim == 1
        if squeeze:
            field_bar = field_bar[:, None]
        nh = self.grid.nlat_half
        fN, fS = self.fourier_analysis(field_bar)
        f = self.adjoint_scale()[:, :, None] / self.solid_angles[:nh, None, None]
        if unscale_coslat:
            f = f / self.coslat[:nh, None, None]
        out = self.legendre_analysis(fN * f, fS * f)
        return out[:, 0] if squeeze else out

    def analyze_adjoint(self, coeffs_bar):
        """grid2spec_pullback! (SpeedyTransformsEnzymeExt.jl:294-323): inverse Legendre,
        times the solid angle, divided by the adjoint scale, then the inverse FFT."""
        coeffs_bar = np.asarray(coeffs_bar, dtype=np.complex128)
        squeeze = coeffs_bar.ndim == 1
        if squeeze:
            coeffs_bar = coeffs_bar[:, None]
        nh = self.grid.nlat_half
        gN, gS = self.legendre_synthesis(coeffs_bar)
        sc = self.adjoint_scale()
        f = np.where(sc > 0, self.solid_angles[:nh, None] / np.where(sc > 0, sc, 1.0), 0.0)[:, :, None]
        out = self.fourier_synthesis(gN * f, gS * f)
        return out[:, 0] if squeeze else out

# ----------------------------------------------------------------------------------------
# gradient arrays (gradient_arrays.jl) -- all indexed by packed lm, 0-based l, m
# ----------------------------------------------------------------------------------------
def _eps(l, m):
    l = np.asarray(l, dtype=np.float64)
    m = np.asarray(m, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.sqrt((l * l - m * m) / (4 * l * l - 1))           # gradient_arrays.jl:4


def gradient_arrays(sp: Spectrum):
    """Return dict of per-lm factors (gradient_arrays.jl:29-145), FP64."""
    l = sp.l_indices.astype(np.float64)
    m = sp.m_indices.astype(np.float64)
    L1 = l + 1   # 1-based degree
    eps_l = _eps(l, m)          # eps at (l, m)     == eps_lm[l,m] 1-based with l->l-1
    eps_lp = _eps(l + 1, m)     # eps at (l+1, m)
    last = np.zeros(sp.nlm, dtype=bool)
    for mm in range(sp.mmax):
        last[sp.offset(mm) + sp.lmax - mm - 1] = True
    grad_y1 = -(L1 - 2) * eps_l
    grad_y2 = np.where(last, 0.0, (L1 + 1) * eps_lp)
    grad_y_vordiv1 = np.where(last, 0.0, L1 * eps_l)
    grad_y_vordiv2 = np.where(last, 0.0, (L1 - 1) * eps_lp)
    grad_x_vordiv = np.where(last, 0.0, m)
    with np.errstate(invalid="ignore", divide="ignore"):
        vordiv_to_uv_x = -m / (L1 * (L1 - 1))
        vordiv_to_uv1 = eps_l / (L1 - 1)
        vordiv_to_uv2 = np.where(last, 0.0, eps_lp / L1)
    vordiv_to_uv_x[0] = 0.0
    vordiv_to_uv1[0] = 0.0
    grad_y1 = np.nan_to_num(grad_y1)
    return dict(grad_y1=grad_y1, grad_y2=grad_y2, grad_y_vordiv1=grad_y_vordiv1,
                grad_y_vordiv2=grad_y_vordiv2, grad_x_vordiv=grad_x_vordiv,
                vordiv_to_uv_x=vordiv_to_uv_x, vordiv_to_uv1=vordiv_to_uv1,
                vordiv_to_uv2=vordiv_to_uv2)


def _shift(a, d):
    """a[lm + d] along axis 0 with zero fill (only used where the factor is zero anyway)."""
    out = np.zeros_like(a)
    if d > 0:
        out[:-d] = a[d:]
    else:
        out[-d:] = a[:d]
    return out


def divergence(sp: Spectrum, u, v, flipsign=False, add=False, out=None, radius=1.0, curl=False):
    """spectral_gradients.jl:83-125 (curl = divergence with u, v swapped and mode=curl)."""
    g = gradient_arrays(sp)
    if curl:
        u, v = v, u
    u = np.asarray(u, dtype=np.complex128)
    v = np.asarray(v, dtype=np.complex128)
    shp = (-1,) + (1,) * (u.ndim - 1)
    mfac = g["grad_x_vordiv"].reshape(shp)
    a = 1j * mfac * u
    b = g["grad_y_vordiv1"].reshape(shp) * _shift(v, -1)
    c = g["grad_y_vordiv2"].reshape(shp) * _shift(v, +1)
    base = (a + b - c) if curl else (a - b + c)
    # lm == 1 (0-based 0): kernel_func(div, 0, 0, grad_y_vordiv2[1] * v[2])
    first = g["grad_y_vordiv2"][0] * v[1]
    base[0] = (-first) if curl else first
    base[sp.nlm - 1] = 0.0       # lm == lmmax writes 0 irrespective of add/flipsign
    val = -base if flipsign else base
    if add:
        if out is None:
            raise ValueError("add=True needs out")
        res = out + val
    else:
        res = val
    res[sp.nlm - 1] = 0.0
    if radius != 1:
        res = res / radius
    return res


def curl(sp, u, v, **kw):
    return divergence(sp, u, v, curl=True, **kw)


def UV_from_vordiv(sp: Spectrum, vor, div=None, radius=1.0):
    """spectral_gradients.jl:269-366. With div=None: UV_from_vor."""
    g = gradient_arrays(sp)
    vor = np.asarray(vor, dtype=np.complex128)
    shp = (-1,) + (1,) * (vor.ndim - 1)
    z = 1j * g["vordiv_to_uv_x"].reshape(shp)
    u1 = g["vordiv_to_uv1"].reshape(shp)
    u2 = g["vordiv_to_uv2"].reshape(shp)
    l = sp.l_indices
    second_last = (l + 1) == (sp.lmax - 1)
    last = (l + 1) == sp.lmax
    vm, vp = _shift(vor, -1), _shift(vor, +1)
    if div is None:
        U = u2 * vp - u1 * vm
        V = z * vor
        U[second_last] = (-u1 * vm)[second_last]
        U[last] = (-u1 * vm)[last]
        V[last] = 0.0
        U[0] = u2[0] * vor[1]
        V[0] = z[0] * vor[0]
    else:
        div = np.asarray(div, dtype=np.complex128)
        dm, dp = _shift(div, -1), _shift(div, +1)
        dzt = u2 * vp - u1 * vm
        ddt = u1 * dm - u2 * dp
        U = z * div + dzt
        V = z * vor + ddt
        U[second_last] = (z * div - u1 * vm)[second_last]
        V[second_last] = (z * vor + u1 * dm)[second_last]
        U[last] = (-u1 * vm)[last]
        V[last] = (u1 * dm)[last]
        U[0] = (z[0] * div[0] + u2[0] * vor[1])
        V[0] = (z[0] * vor[0] - u2[0] * div[1])
    if radius != 1:
        U = U * radius
        V = V * radius
    return U, V


def laplace(sp: Spectrum, alms, inverse=False, flipsign=False, add=False, out=None, radius=1.0):
    """spectral_gradients.jl:386-421."""
    ev = -(np.arange(sp.lmax) * (np.arange(sp.lmax) + 1.0))
    if inverse:
        e = np.zeros_like(ev)
        e[1:] = 1.0 / ev[1:]
        ev = e
    alms = np.asarray(alms, dtype=np.complex128)
    shp = (-1,) + (1,) * (alms.ndim - 1)
    a = alms * ev[sp.l_indices].reshape(shp)
    a = -a if flipsign else a
    res = (out + a) if add else a
    if radius != 1:
        res = res * (radius ** 2 if inverse else 1.0 / radius ** 2)
    return res


def gradient(sp: Spectrum, p, radius=1.0):
    """spectral_gradients.jl:483-527: returns (dpdx, dpdy)."""
    g = gradient_arrays(sp)
    p = np.asarray(p, dtype=np.complex128)
    shp = (-1,) + (1,) * (p.ndim - 1)
    dpdx = 1j * sp.m_indices.reshape(shp) * p
    gy1 = g["grad_y1"].reshape(shp)
    gy2 = g["grad_y2"].reshape(shp)
    dpdy = gy1 * _shift(p, -1) + gy2 * _shift(p, +1)
    dpdy[0] = gy2[0] * p[1]
    dpdy[sp.nlm - 1] = gy1[sp.nlm - 1] * p[sp.nlm - 2]
    if radius != 1:
        dpdx = dpdx / radius
        dpdy = dpdy / radius
    return dpdx, dpdy


# ----------------------------------------------------------------------------------------
# seeded synthetic inputs (shapes and distributions of the benchmark configurations)
# ----------------------------------------------------------------------------------------
def random_coeffs(sp: Spectrum, K: int, seed: int = 0, zero_last_degree: bool = False):
    """Re, Im ~ N(0,1) (l+1)^-1.5, Im(m=0) = 0; optionally zero the last degree row."""
    rng = np.random.default_rng(seed)
    re = rng.standard_normal((sp.nlm, K))
    im = rng.standard_normal((sp.nlm, K))
    scale = (sp.l_indices + 1.0) ** -1.5
    c = (re + 1j * im) * scale[:, None]
    c[sp.m_indices == 0] = c[sp.m_indices == 0].real
    if zero_last_degree:
        for m in range(sp.mmax):
            c[sp.offset(m) + sp.lmax - m - 1] = 0.0
    return c


def rel_err(x, ref):
    x = np.asarray(x)
    ref = np.asarray(ref)
    return float(np.linalg.norm((x - ref).ravel()) / max(np.linalg.norm(ref.ravel()), 1e-300))
