"""GPU parity: libsht's CUDA kernels (through the C ABI) against the FP64 oracle.

Mirrors SpeedyWeather/test/GPU/spectral_transform.jl (GPU vs CPU at
rtol = sqrt(eps(Float32)), outputs pre-filled with NaN so a missing write shows)
and the invariants of SpeedyTransforms/test/spectral_transform.jl.
Tolerance: relative L2 error <= 1e-5 against FP64 for the FP32 path.
"""
import math

import numpy as np
import pytest

import sht_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def st():
    import torch  # noqa: F401
    import speedytransforms as st
    return st


_cache = {}


def setup(st, T, grid, K, one_more=False, precision="fp32", nh=None, shortcut="linear"):
    key = (T, grid, K, one_more, precision, nh, shortcut)
    if key in _cache:
        return _cache[key]
    nh = nh or O.get_nlat_half(T)
    kind = O.FULL_GAUSSIAN if grid == "full" else O.OCTAHEDRAL_GAUSSIAN
    sp = st.Spectrum(T + int(one_more), T)
    G = st.FullGaussianGrid if grid == "full" else st.OctahedralGaussianGrid
    S = st.SpectralTransform(sp, G(nh), nlayers=K, precision=precision, LegendreShortcut=shortcut)
    So = O.SpectralTransform(O.Spectrum(T + int(one_more), T), O.Grid(kind, nh), shortcut=shortcut)
    _cache[key] = (S, So)
    return S, So


def to_lta(st, S, c):
    import torch
    t = torch.tensor(np.ascontiguousarray(c.T), dtype=torch.complex64, device="cuda")
    return st.LowerTriangularArray(t, S.spectrum)


def to_field(st, S, f):
    import torch
    t = torch.tensor(np.ascontiguousarray(f.T), dtype=torch.float32, device="cuda")
    return st.Field(t, S.grid)


def np_of(x):
    import torch
    torch.cuda.synchronize()
    return x.data.cpu().numpy().T.astype(np.complex128 if x.data.is_complex() else np.float64)


def nan_field(st, S, K):
    import torch
    return st.Field(torch.full((K, S.grid.npoints), float("nan"), device="cuda"), S.grid)


def nan_lta(st, S, K):
    import torch
    return st.LowerTriangularArray(torch.full((K, S.spectrum.nlm), complex("nan+nanj"), dtype=torch.complex64,
                                              device="cuda"), S.spectrum)


CASES = [(31, "full", 8), (31, "octa", 8), (63, "octa", 8), (127, "octa", 48)]


@pytest.mark.parametrize("T,grid,K", CASES)
def test_synthesis_matches_oracle(st, T, grid, K):
    S, So = setup(st, T, grid, K)
    c = O.random_coeffs(So.spectrum, K, seed=T)
    f = nan_field(st, S, K)
    st.transform_(f, to_lta(st, S, c), S)
    got = np_of(f)
    assert np.all(np.isfinite(got)), "synthesis left unwritten (NaN) grid points"
    ref = So.synthesize(c)
    assert O.rel_err(got, ref) < TOL


@pytest.mark.parametrize("T,grid,K", CASES)
def test_analysis_matches_oracle(st, T, grid, K):
    S, So = setup(st, T, grid, K)
    c = O.random_coeffs(So.spectrum, K, seed=T + 1)
    f = So.synthesize(c)                       # band-limited grid input
    out = nan_lta(st, S, K)
    st.transform_(out, to_field(st, S, f.astype(np.float32)), S)
    got = np_of(out)
    assert np.all(np.isfinite(got)), "analysis left unwritten (NaN) coefficients"
    ref = So.analyze(f.astype(np.float32).astype(np.float64))
    assert O.rel_err(got, ref) < TOL


@pytest.mark.parametrize("T,grid,K", CASES[:3])
def test_roundtrip_bandlimited(st, T, grid, K):
    S, So = setup(st, T, grid, K)
    c = O.random_coeffs(So.spectrum, K, seed=7)
    lt = to_lta(st, S, c)
    f = st.transform(lt, S)
    c2 = st.transform(f, S)
    ref = So.analyze(So.synthesize(c))
    assert O.rel_err(np_of(c2), ref) < TOL


def test_a00_constant(st):
    # spectral_transform.jl:38-69 on the GPU path
    for grid in ("full", "octa"):
        S, So = setup(st, 31, grid, 8)
        c = np.zeros((So.spectrum.nlm, 1), complex)
        c[0] = 2 * math.sqrt(math.pi)
        f = st.transform(to_lta(st, S, c[:, 0]), S)
        np.testing.assert_allclose(np_of(f), 1.0, rtol=2e-6)


def test_individual_harmonics(st):
    # spectral_transform.jl:71-102: atol = 100 eps(Float32)
    S, So = setup(st, 31, "octa", 8)
    sp = So.spectrum
    for l in range(3):
        for m in range(l + 1):
            a = np.zeros(sp.nlm, complex)
            a[sp.lm(l, m)] = 1
            a2 = np_of(st.transform(st.transform(to_lta(st, S, a), S), S))
            ref = a.copy()
            ref[sp.m_indices == 0] = ref[sp.m_indices == 0].real
            np.testing.assert_allclose(a2, ref, atol=100 * np.finfo(np.float32).eps)


def test_singleton_layer_bitwise(st):
    # spectral_transform.jl:104-156: a single layer equals the same layer of a batch, bitwise
    S, So = setup(st, 63, "octa", 8)
    c = O.random_coeffs(So.spectrum, 8, seed=3)
    fb = np_of(st.transform(to_lta(st, S, c), S))
    f1 = np_of(st.transform(to_lta(st, S, c[:, 2]), S))
    np.testing.assert_array_equal(f1, fb[:, 2])
    g = fb.astype(np.float32)
    cb = np_of(st.transform(to_field(st, S, g), S))
    c1 = np_of(st.transform(to_field(st, S, g[:, 5]), S))
    np.testing.assert_array_equal(c1, cb[:, 5])


def test_unscale_coslat_and_add(st):
    import torch
    S, So = setup(st, 63, "octa", 8)
    c = O.random_coeffs(So.spectrum, 4, seed=11)
    lt = to_lta(st, S, c)
    f = st.transform(lt, S, unscale_coslat=True)
    ref = So.synthesize(c, unscale_coslat=True)
    assert O.rel_err(np_of(f), ref) < TOL
    base = torch.randn(4, S.grid.npoints, device="cuda")
    f2 = st.Field(base.clone(), S.grid)
    st.transform_(f2, lt, S, add=True)
    assert O.rel_err(np_of(f2), So.synthesize(c) + base.cpu().numpy().T) < TOL
    out = st.transform(f2, S)
    acc = st.LowerTriangularArray(out.data.clone(), S.spectrum)
    st.transform_(acc, f2, S, add=True)
    np.testing.assert_allclose(np_of(acc), 2 * np_of(out), rtol=1e-6, atol=1e-7)


def test_split_stages_equal_fused(st):
    import torch
    from speedytransforms import _lib
    S, So = setup(st, 63, "octa", 8)
    c = O.random_coeffs(So.spectrum, 8, seed=4)
    lt = to_lta(st, S, c)
    f = st.transform(lt, S)
    f2 = torch.empty_like(f.data)
    sp = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib.sht_legendre_synthesis(S.handle, lt.data.data_ptr(), S.spectrum.nlm, 8, sp))
    _lib.check(_lib.lib.sht_fourier_synthesis(S.handle, f2.data_ptr(), S.grid.npoints, 8, 0, sp))
    torch.cuda.synchronize()
    assert torch.equal(f.data, f2)


def test_strided_views(st):
    # fields and coefficients as row views of larger parents (the reference's fused parents)
    import torch
    S, So = setup(st, 31, "octa", 8)
    c = O.random_coeffs(So.spectrum, 3, seed=9)
    parent = torch.zeros(6, S.spectrum.nlm + 17, dtype=torch.complex64, device="cuda")
    parent[1:4, :S.spectrum.nlm] = torch.tensor(c.T, dtype=torch.complex64, device="cuda")
    lt = st.LowerTriangularArray(parent[1:4, :S.spectrum.nlm], S.spectrum)
    gparent = torch.full((5, S.grid.npoints + 5), 7.0, device="cuda")
    f = st.Field(gparent[1:4, :S.grid.npoints], S.grid)
    st.transform_(f, lt, S)
    assert O.rel_err(np_of(f), So.synthesize(c)) < TOL
    assert torch.all(gparent[0] == 7.0) and torch.all(gparent[4] == 7.0)
    assert torch.all(gparent[1:4, S.grid.npoints:] == 7.0)


def test_dimension_mismatch(st):
    S, So = setup(st, 31, "octa", 8)
    S2, _ = setup(st, 63, "octa", 8)
    c = to_lta(st, S, O.random_coeffs(So.spectrum, 2))
    with pytest.raises(st.DimensionMismatch):
        st.transform_(st.Field.zeros(S2.grid, 2), c, S)
    big = to_lta(st, S, O.random_coeffs(So.spectrum, 9))
    with pytest.raises(st.DimensionMismatch):
        st.transform(big, S)


@pytest.mark.parametrize("shortcut", ["quadratic", "cubic", "linquadcoslat2", "lincubcoslat"])
def test_other_shortcuts(st, shortcut):
    S, So = setup(st, 63, "octa", 4, shortcut=shortcut)
    c = O.random_coeffs(So.spectrum, 4, seed=12)
    f = st.transform(to_lta(st, S, c), S)
    assert O.rel_err(np_of(f), So.synthesize(c)) < TOL
    g = So.synthesize(c).astype(np.float32)
    out = st.transform(to_field(st, S, g), S)
    assert O.rel_err(np_of(out), So.analyze(g.astype(np.float64))) < TOL


# ------------------------------ operators --------------------------------------------------
def _ops_setup(st):
    S, So = setup(st, 31, "octa", 4, one_more=True)
    sp = So.spectrum
    rng = np.random.default_rng(21)
    mk = lambda: rng.standard_normal((sp.nlm, 4)) + 1j * rng.standard_normal((sp.nlm, 4))
    return S, So, sp, mk


def test_divergence_curl_match_oracle(st):
    S, So, sp, mk = _ops_setup(st)
    u, v, o = mk(), mk(), mk()
    for fn, ofn in ((st.divergence_, O.divergence), (st.curl_, O.curl)):
        for flip in (False, True):
            for add in (False, True):
                for radius in (1.0, 6.371e6):
                    out = to_lta(st, S, o)
                    fn(out, to_lta(st, S, u), to_lta(st, S, v), S, flipsign=flip, add=add, radius=radius)
                    ref = ofn(sp, u, v, flipsign=flip, add=add, out=o.copy(), radius=radius)
                    assert O.rel_err(np_of(out), ref) < TOL


def test_uv_from_vordiv_match_oracle(st):
    S, So, sp, mk = _ops_setup(st)
    vor, div = mk(), mk()
    for radius in (1.0, 6.371e6):
        U, V = st.UV_from_vordiv(to_lta(st, S, vor), to_lta(st, S, div), S, radius=radius)
        Ur, Vr = O.UV_from_vordiv(sp, vor, div, radius=radius)
        assert O.rel_err(np_of(U), Ur) < TOL and O.rel_err(np_of(V), Vr) < TOL
        U, V = st.UV_from_vor(to_lta(st, S, vor), S, radius=radius)
        Ur, Vr = O.UV_from_vordiv(sp, vor, radius=radius)
        assert O.rel_err(np_of(U), Ur) < TOL and O.rel_err(np_of(V), Vr) < TOL


def test_laplace_gradient_match_oracle(st):
    S, So, sp, mk = _ops_setup(st)
    a, o = mk(), mk()
    for inv in (False, True):
        for flip in (False, True):
            for add in (False, True):
                out = to_lta(st, S, o)
                st.laplace_(out, to_lta(st, S, a), S, inverse=inv, flipsign=flip, add=add, radius=2.0)
                ref = O.laplace(sp, a, inverse=inv, flipsign=flip, add=add, out=o.copy(), radius=2.0)
                assert O.rel_err(np_of(out), ref) < TOL
    dx, dy = st.gradient(to_lta(st, S, a), S, radius=3.0)
    rx, ry = O.gradient(sp, a, radius=3.0)
    assert O.rel_err(np_of(dx), rx) < TOL and O.rel_err(np_of(dy), ry) < TOL


def test_operators_layer_groups_match_oracle(st):
    """At T255 with 22 layers the operator kernels run several layers per thread (8 for
    curl/divergence, the Laplacians and the gradient, 4 for UV_from_vordiv) with a partial
    last group (22 = 8 + 8 + 6 = 5 x 4 + 2); outputs NaN-prefilled, every flag."""
    import torch
    K = 22
    S, So = setup(st, 255, "octa", K, one_more=True)
    sp = So.spectrum
    rng = np.random.default_rng(8)
    mk = lambda: rng.standard_normal((sp.nlm, K)) + 1j * rng.standard_normal((sp.nlm, K))
    u, v, o = mk(), mk(), mk()

    def nan_lta():
        return st.LowerTriangularArray(torch.full((K, sp.nlm), complex(np.nan, np.nan), dtype=torch.complex64,
                                                  device="cuda"), S.spectrum)
    for fn, ofn in ((st.divergence_, O.divergence), (st.curl_, O.curl)):
        for flip, add in ((False, False), (True, True)):
            out = to_lta(st, S, o) if add else nan_lta()
            fn(out, to_lta(st, S, u), to_lta(st, S, v), S, flipsign=flip, add=add, radius=6.371e6)
            ref = ofn(sp, u, v, flipsign=flip, add=add, out=o.copy(), radius=6.371e6)
            assert O.rel_err(np_of(out), ref) < TOL
    U, V = nan_lta(), nan_lta()
    st.UV_from_vordiv_(U, V, to_lta(st, S, u), to_lta(st, S, v), S, radius=6.371e6)
    Ur, Vr = O.UV_from_vordiv(sp, u, v, radius=6.371e6)
    assert O.rel_err(np_of(U), Ur) < TOL and O.rel_err(np_of(V), Vr) < TOL
    U, V = nan_lta(), nan_lta()
    st.UV_from_vor_(U, V, to_lta(st, S, u), S)
    Ur, Vr = O.UV_from_vordiv(sp, u)
    assert O.rel_err(np_of(U), Ur) < TOL and O.rel_err(np_of(V), Vr) < TOL
    for inv in (False, True):
        for flip, add in ((False, False), (True, True)):
            out = to_lta(st, S, o) if add else nan_lta()
            st.laplace_(out, to_lta(st, S, u), S, inverse=inv, flipsign=flip, add=add, radius=2.0)
            ref = O.laplace(sp, u, inverse=inv, flipsign=flip, add=add, out=o.copy(), radius=2.0)
            assert O.rel_err(np_of(out), ref) < TOL
    dx, dy = nan_lta(), nan_lta()
    st.gradient_(dx, dy, to_lta(st, S, u), S, radius=3.0)
    rx, ry = O.gradient(sp, u, radius=3.0)
    assert O.rel_err(np_of(dx), rx) < TOL and O.rel_err(np_of(dy), ry) < TOL
    assert S.device_status() == 0


def test_vordiv_uv_roundtrip_gpu(st):
    # spectral_gradients.jl tests :201-252 on the GPU path (Float32: rtol = 80 sqrt(eps(Float32)))
    import torch
    S, So = setup(st, 32, "octa", 2, one_more=True)
    sp = So.spectrum
    rng = np.random.default_rng(5)
    vor = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    div = rng.standard_normal((sp.nlm, 2)) + 1j * rng.standard_normal((sp.nlm, 2))
    for a in (vor, div):
        for m in range(sp.mmax):
            a[sp.offset(m) + sp.lmax - m - 1] = 0
        a[0] = 0
        a[sp.m_indices == 0] = a[sp.m_indices == 0].real
    U, V = st.UV_from_vordiv(to_lta(st, S, vor), to_lta(st, S, div), S)
    u = st.transform(U, S, unscale_coslat=True)
    v = st.transform(V, S, unscale_coslat=True)
    c = torch.tensor(1.0 / np.cos(np.radians(S.latd)), dtype=torch.float32, device="cuda")
    c = torch.repeat_interleave(c, torch.tensor(S.grid.nlons, device="cuda"))
    u.data *= c
    v.data *= c
    uh, vh = st.transform(u, S), st.transform(v, S)
    tol = 80 * math.sqrt(np.finfo(np.float32).eps)
    np.testing.assert_allclose(np_of(st.curl(uh, vh, S)), vor, rtol=tol, atol=tol)
    np.testing.assert_allclose(np_of(st.divergence(uh, vh, S)), div, rtol=tol, atol=tol)


# ------------------------------ full size (T511 x 64) -------------------------------------
def test_t511_full_size_parity(st):
    """Synthesis and analysis at the benchmark size, against FP64 on a subset of layers
    and through size-independent properties on all 64 layers."""
    S, So = setup(st, 512, "octa", 64, nh=384)
    sp = So.spectrum
    c = O.random_coeffs(sp, 64, seed=2)
    lt = to_lta(st, S, c)
    f = st.transform(lt, S)
    fg = np_of(f)
    assert np.all(np.isfinite(fg))
    sub = [0, 37, 63]
    ref = So.synthesize(c[:, sub])
    assert O.rel_err(fg[:, sub], ref) < TOL
    c2 = st.transform(f, S)
    refc = So.analyze(fg[:, sub].astype(np.float32).astype(np.float64))
    assert O.rel_err(np_of(c2)[:, sub], refc) < TOL
    # linearity on all layers: T(a + 2b) = T(a) + 2 T(b)
    import torch
    lt2 = st.LowerTriangularArray(lt.data + 2 * torch.roll(lt.data, 1, 0), S.spectrum)
    f2 = st.transform(lt2, S)
    lin = f.data + 2 * torch.roll(f.data, 1, 0)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(f2.data - lin) / torch.linalg.norm(lin)) < TOL


def _isapprox(x, y, atol, rtol):
    """Julia's elementwise x ≈ y (atol, rtol): |x - y| <= max(atol, rtol max(|x|, |y|))."""
    return np.all(np.abs(x - y) <= np.maximum(atol, rtol * np.maximum(np.abs(x), np.abs(y))))


@pytest.mark.parametrize("grid", ["full", "octa"])
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_idempotence_orography(st, grid, precision):
    """spectral_transform.jl:281-324 ("Transform: Orography (exact grids)"): a rough field
    (5000 rand^2), analysed, band-limited (here sharply, degrees above 0.95 T removed, where
    the reference uses spectral_smoothing), then synthesised and analysed twice: both
    passes agree to 2 sqrt(eps(Float32)) elementwise. Split-BF16 plans carry ~1e-5
    relative error, so their absolute tolerance scales with the field's maximum."""
    import torch
    T = 32
    S, So = setup(st, T, grid, 1, precision=precision, nh=O.get_nlat_half(T, 2))
    rng = np.random.default_rng(3)
    oro = (5000 * rng.random(S.grid.npoints) ** 2)[:, None]
    f0 = to_field(st, S, oro)
    spec = st.transform(f0, S)
    t = round(T * 0.95)
    keep = torch.tensor(So.spectrum.l_indices <= t, device="cuda")
    spec.data[:, ~keep] = 0
    grid1 = st.transform(spec, S)
    spec1 = st.transform(grid1, S)
    grid2 = st.transform(spec1, S)
    spec2 = st.transform(grid2, S)
    tol = 2 * math.sqrt(np.finfo(np.float32).eps)
    g1, g2, s1, s2 = np_of(grid1), np_of(grid2), np_of(spec1), np_of(spec2)
    atol_g = tol if precision == "fp32" else tol * np.abs(g1).max()
    atol_s = tol if precision == "fp32" else tol * np.abs(s1).max()
    assert _isapprox(g1, g2, atol_g, tol)
    assert _isapprox(s1, s2, atol_s, tol)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_roundtrip_every_layer_count(st, precision):
    """spectral_transform.jl:375-407: a transform planned for 4 layers runs K = 1, 2, 3, 4
    (no per-K plans are needed here: every launch takes K) and spec -> grid -> spec -> grid
    reproduces the grid (relative L2 1e-5 in FP32; the reference's 1e-13 is for Float64)."""
    import torch
    T = 32
    S, So = setup(st, T, "full", 4, precision=precision, nh=O.get_nlat_half(T, 3))
    for K in (1, 2, 3, 4):
        g = torch.Generator().manual_seed(K)
        c = torch.complex(torch.randn(K, S.spectrum.nlm, generator=g), torch.randn(K, S.spectrum.nlm, generator=g))
        spec_in = st.LowerTriangularArray(c.to(torch.complex64).cuda(), S.spectrum)
        grid_out = st.transform(spec_in, S)
        spec_back = st.transform(grid_out, S)
        grid_back = st.transform(spec_back, S)
        a, b = np_of(grid_back), np_of(grid_out)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < TOL, K
