"""Pins the FP64 oracle against the reference's own known answers and invariant tests.

Mirrors SpeedyTransforms/test/spectral_transform.jl and
SpeedyTransforms/test/spectral_gradients.jl on the oracle (CPU only).
"""
import math

import numpy as np
import pytest

import sht_oracle as O


def make(T, kind, dealiasing=2.0, one_more=False):
    sp = O.Spectrum(T + int(one_more), T)
    g = O.Grid(kind, O.get_nlat_half(T, dealiasing))
    return sp, g, O.SpectralTransform(sp, g)


def test_resolution_match():
    # spectral_transform.jl:1-30
    for dealiasing in (2, 3):
        for i in range(5, 11):
            T = 2 ** i
            nh = O.get_nlat_half(T, dealiasing)
            assert (4 * nh, 2 * nh) == ((dealiasing + 1) * 2 ** i, (dealiasing + 1) * 2 ** i // 2)
            assert O.get_truncation(nh, dealiasing) == T


def test_gauss_legendre_matches_numpy():
    for n in (48, 96, 192, 768):
        x, w = O.gauss_legendre(n)
        x2, w2 = np.polynomial.legendre.leggauss(n)
        assert np.max(np.abs(x - x2)) < 1e-14
        assert np.max(np.abs(w - w2)) < 1e-13
        assert abs(w.sum() - 2.0) < 1e-13


def test_legendre_closed_forms():
    x = np.array([0.31, -0.7, 0.95, 0.0])
    sp = O.Spectrum(4, 4)
    lam = O.legendre_table(sp, x)
    s = np.sqrt(1 - x * x)
    pi = math.pi
    ref = {(0, 0): np.full_like(x, 1 / (2 * math.sqrt(pi))),
           (1, 0): math.sqrt(3 / (4 * pi)) * x,
           (1, 1): -math.sqrt(3 / (8 * pi)) * s,
           (2, 0): math.sqrt(5 / (16 * pi)) * (3 * x * x - 1),
           (2, 1): -math.sqrt(15 / (8 * pi)) * x * s,
           (2, 2): math.sqrt(15 / (32 * pi)) * s * s,
           (3, 3): -math.sqrt(35 / (64 * pi)) * s ** 3}
    for (l, m), v in ref.items():
        np.testing.assert_allclose(lam[sp.lm(l, m)], v, atol=1e-15)


@pytest.mark.parametrize("kind", [O.FULL_GAUSSIAN, O.OCTAHEDRAL_GAUSSIAN])
@pytest.mark.parametrize("T", [32, 64])
def test_a00_constant(kind, T):
    # spectral_transform.jl:38-69 and spectral_transform.jl:158 (norm_sphere = 2 sqrt(pi))
    sp, g, S = make(T, kind)
    a = np.zeros(sp.nlm, complex)
    a[0] = 1
    f = S.synthesize(a)
    assert np.all(f > 0)
    np.testing.assert_allclose(f, f[0], rtol=1e-14)
    a[0] = S.norm_sphere
    np.testing.assert_allclose(S.synthesize(a), 1.0, rtol=1e-14)


@pytest.mark.parametrize("kind", [O.FULL_GAUSSIAN, O.OCTAHEDRAL_GAUSSIAN])
@pytest.mark.parametrize("T", [32, 64])
def test_individual_harmonics_roundtrip(kind, T):
    # spectral_transform.jl:71-102 (atol = 100 eps(Float64))
    sp, g, S = make(T, kind)
    for l in range(3):
        for m in range(l + 1):
            a = np.zeros(sp.nlm, complex)
            a[sp.lm(l, m)] = 1
            a2 = S.analyze(S.synthesize(a))
            ref = a.copy()
            ref[sp.m_indices == 0] = ref[sp.m_indices == 0].real
            np.testing.assert_allclose(a2, ref, atol=100 * np.finfo(float).eps)


@pytest.mark.parametrize("kind", [O.FULL_GAUSSIAN, O.OCTAHEDRAL_GAUSSIAN])
@pytest.mark.parametrize("T", [43, 64])
def test_roundtrip_accuracy(kind, T):
    # spectral_transform.jl:326-373: dealiasing 3, Float64, 8 layers, rtol 1e-13 (Gaussian grids)
    sp, g, S = make(T, kind, dealiasing=3)
    rng = np.random.default_rng(0)
    spec = rng.standard_normal((sp.nlm, 8)) + 1j * rng.standard_normal((sp.nlm, 8))
    grid = S.synthesize(spec)
    grid2 = S.synthesize(S.analyze(grid))
    assert O.rel_err(grid2, grid) < 1e-13


def test_set_constant_known_answer():
    # SpeedyWeather/src/variables/set.jl:145-152: a_00 = c 2 sqrt(pi) gives a grid of c
    sp, g, S = make(31, O.OCTAHEDRAL_GAUSSIAN)
    a = np.zeros(sp.nlm, complex)
    a[0] = 287.5 * 2 * math.sqrt(math.pi)
    np.testing.assert_allclose(S.synthesize(a), 287.5, rtol=1e-13)
    c = S.analyze(np.full(g.npoints, 287.5))
    assert abs(c[0] - 287.5 * 2 * math.sqrt(math.pi)) < 1e-9
    assert np.max(np.abs(c[1:])) < 1e-9


# ------------------------------ operators (spectral_gradients.jl tests) ----------------
def _vector_setup(T=32, seed=0):
    sp = O.Spectrum(T + 1, T)
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((sp.nlm, 3)) + 1j * rng.standard_normal((sp.nlm, 3))
    a[sp.m_indices == 0] = a[sp.m_indices == 0].real
    for m in range(sp.mmax):
        a[sp.offset(m) + sp.lmax - m - 1] = 0
    return sp, a


def _uv_chain(S, U, V):
    """U, V -> grid with unscale_coslat -> scale_coslat^-1 -> spectral (the reference tests' chain)."""
    nh = S.grid.nlat_half
    c = 1.0 / S.grid.coslat[S.grid.whichring()]
    u = S.synthesize(U, unscale_coslat=True) * c[:, None]
    v = S.synthesize(V, unscale_coslat=True) * c[:, None]
    del nh
    return S.analyze(u), S.analyze(v)


def test_div_of_nondivergent_is_zero():
    # spectral_gradients.jl tests :1-52 (compares the divergence it computes with zero)
    sp, g, S = make(31, O.OCTAHEDRAL_GAUSSIAN, one_more=True)
    rng = np.random.default_rng(0)
    vor = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    U, V = O.UV_from_vordiv(sp, vor, np.zeros_like(vor))
    U2, V2 = O.UV_from_vordiv(sp, vor)
    np.testing.assert_array_equal(S.synthesize(U, True), S.synthesize(U2, True))
    np.testing.assert_array_equal(S.synthesize(V, True), S.synthesize(V2, True))
    uh, vh = _uv_chain(S, U, V)
    assert np.max(np.abs(O.divergence(sp, uh, vh))) < math.sqrt(np.finfo(float).eps)


def test_curl_of_irrotational_is_zero():
    # spectral_gradients.jl tests :54-94
    sp, g, S = make(32, O.OCTAHEDRAL_GAUSSIAN, one_more=True)
    rng = np.random.default_rng(1)
    div = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    U, V = O.UV_from_vordiv(sp, np.zeros_like(div), div)
    uh, vh = _uv_chain(S, U, V)
    assert np.max(np.abs(O.curl(sp, uh, vh))) < math.sqrt(np.finfo(float).eps)


def test_vordiv_uv_roundtrip():
    # spectral_gradients.jl tests :201-252, rtol = 80 sqrt(eps)
    sp, g, S = make(32, O.OCTAHEDRAL_GAUSSIAN, one_more=True)
    rng = np.random.default_rng(2)
    vor = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    div = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    for a in (vor, div):
        for m in range(sp.mmax):
            a[sp.offset(m) + sp.lmax - m - 1] = 0
        a[0] = 0
        a[sp.m_indices == 0] = a[sp.m_indices == 0].real
    U, V = O.UV_from_vordiv(sp, vor, div)
    uh, vh = _uv_chain(S, U, V)
    tol = 80 * math.sqrt(np.finfo(float).eps)
    np.testing.assert_allclose(O.curl(sp, uh, vh), vor, rtol=tol, atol=tol)
    np.testing.assert_allclose(O.divergence(sp, uh, vh), div, rtol=tol, atol=tol)


def test_curl_grad_zero_div_grad_laplace():
    # spectral_gradients.jl tests :306-346 (FullGaussianGrid, tol 5 sqrt(eps))
    sp, g, S = make(32, O.FULL_GAUSSIAN, one_more=True)
    rng = np.random.default_rng(3)
    a = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    for m in range(sp.mmax):
        a[sp.offset(m) + sp.lmax - m - 1] = 0
    a[sp.m_indices == 0] = a[sp.m_indices == 0].real
    dx, dy = O.gradient(sp, a)
    c2 = (1.0 / g.coslat[g.whichring()] ** 2)[:, None]
    dx = S.analyze(S.synthesize(dx) * c2)
    dy = S.analyze(S.synthesize(dy) * c2)
    tol = 5 * math.sqrt(np.finfo(float).eps)
    assert np.max(np.abs(O.curl(sp, dx, dy))) < tol
    np.testing.assert_allclose(O.divergence(sp, dx, dy), O.laplace(sp, a), atol=tol, rtol=tol)


def test_laplace_inverse_identity():
    # spectral_gradients.jl tests :254-304
    sp, a = _vector_setup(seed=4)
    a[0] = 0
    b = O.laplace(sp, O.laplace(sp, a, inverse=True))
    np.testing.assert_allclose(b, a, atol=1e-12)


def test_flipsign_add_semantics():
    # spectral_gradients.jl tests :96-148
    sp, u = _vector_setup(seed=5)
    _, v = _vector_setup(seed=6)
    d = O.divergence(sp, u, v)
    d2 = O.divergence(sp, u, v, flipsign=True)
    np.testing.assert_array_equal(d2, -d)
    d3 = O.divergence(sp, u, v, add=True, out=d)
    np.testing.assert_allclose(d3, 2 * d)


def _rdot(a, b):
    """Real inner product of the Float32 storage: re and im parts as separate reals."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.sum(a.real * b.real) + np.sum(a.imag * b.imag))


@pytest.mark.parametrize("grid", [O.FULL_GAUSSIAN, O.OCTAHEDRAL_GAUSSIAN])
@pytest.mark.parametrize("unscale", [False, True])
def test_adjoint_dot_products(grid, unscale):
    """The restated pullbacks (SpeedyTransformsEnzymeExt.jl:263-323) are the adjoints of
    the transforms: <S c, g> = <c, S^T g> and <A g, c> = <g, A^T c>."""
    T = O.Spectrum(32, 32)
    S = O.SpectralTransform(T, O.Grid(grid, 24))
    rng = np.random.default_rng(7)
    c = rng.standard_normal((T.nlm, 3)) + 1j * rng.standard_normal((T.nlm, 3))
    g = rng.standard_normal((S.grid.npoints, 3))
    lhs = _rdot(S.synthesize(c, unscale_coslat=unscale), g)
    rhs = _rdot(c, S.synthesize_adjoint(g, unscale_coslat=unscale))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1.0)
    lhs = _rdot(S.analyze(g), c)
    rhs = _rdot(g, S.analyze_adjoint(c))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1.0)
