"""Prime-radix first stages of the ring FFTs on the tensor cores (SHT_PRIME_TENSOR).

The tensor-core stage (three TF32 products, FP32 accumulation) and the direct FP32 stage
inside the FFT kernel compute the same DFTs; they agree to FP32 rounding, not bit for bit.
Measured differences between the two modes, relative L2 over the whole output: 0.7e-7
(T127) .. 2.8e-7 (T511 round trip), so the tests allow 1e-6. Against the FP64 oracle both stay at the FP32
plans' level (1e-5 bar of the parity tests).
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import nan_field, nan_lta, np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

MODE_TOL = 1e-6
TOL = 1e-5


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


def _both(S, fn):
    """fn() with the tensor-core first stages, then with the direct ones; the plan's mode
    is restored afterwards."""
    mode = S.prime_stage
    try:
        S.prime_stage = "tensor"
        a = fn()
        assert S.device_status() == 0
        S.prime_stage = "direct"
        b = fn()
        assert S.device_status() == 0
    finally:
        S.prime_stage = mode
    return a, b


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_modes_and_availability(st):
    S, _ = setup(st, 127, "octa", 8, precision="fp16x3")
    assert S.prime_stage_available
    assert S.prime_stage == "direct"          # the default: the FFT kernel's own stage
    S.prime_stage = "tensor"
    assert S.prime_stage == "tensor"
    S.prime_stage = "direct"
    full, _ = setup(st, 31, "full", 4)
    assert not full.prime_stage_available    # 96-point rings: radices 2 and 3 only
    with pytest.raises(ValueError):
        S.prime_stage = "sideways"


@pytest.mark.parametrize("T,K", [(127, 48), (255, 16)])
def test_fp32_plan_tensor_vs_direct_and_oracle(st, T, K):
    """FP32 plan: the prime stage is the only difference between the modes."""
    S, So = setup(st, T, "octa", K)
    assert S.prime_stage_available
    c = O.random_coeffs(So.spectrum, K, seed=T + 11)
    lta = to_lta(st, S, c)

    def syn():
        f = nan_field(st, S, K)
        st.transform_(f, lta, S)
        return np_of(f)

    ft, fd = _both(S, syn)
    assert np.all(np.isfinite(ft))
    assert _rel(ft, fd) < MODE_TOL
    ref = So.synthesize(c)
    assert O.rel_err(ft, ref) < TOL
    g = ref.astype(np.float32)
    field = to_field(st, S, g)

    def ana():
        out = nan_lta(st, S, K)
        st.transform_(out, field, S)
        return np_of(out)

    at, ad = _both(S, ana)
    assert np.all(np.isfinite(at))
    assert _rel(at, ad) < MODE_TOL
    assert O.rel_err(at, So.analyze(g.astype(np.float64))) < TOL


def test_fewer_layers_than_the_plan_and_flags(st):
    """K < nlayers (partial column tiles), unscale_coslat and add in the synthesis."""
    import torch
    S, So = setup(st, 255, "octa", 24)
    K = 7
    c = O.random_coeffs(So.spectrum, K, seed=5)
    lta = to_lta(st, S, c)
    base = torch.randn(K, S.grid.npoints, device="cuda")

    def syn():
        f = st.Field(base.clone(), S.grid)
        st.transform_(f, lta, S, unscale_coslat=True, add=True)
        return np_of(f)

    ft, fd = _both(S, syn)
    assert _rel(ft - base.cpu().numpy().T, fd - base.cpu().numpy().T) < MODE_TOL
    g = So.synthesize(c).astype(np.float32)
    field = to_field(st, S, g)

    def ana():
        out = nan_lta(st, S, K)
        st.transform_(out, field, S)
        return np_of(out)

    at, ad = _both(S, ana)
    assert _rel(at, ad) < MODE_TOL
    assert O.rel_err(at, So.analyze(g.astype(np.float64))) < TOL


def test_adjoints_tensor_vs_direct(st):
    """The pullbacks run the FFT stages with the adjoint weights."""
    import torch
    S, So = setup(st, 127, "octa", 12)
    K = 12
    gbar = to_field(st, S, np.random.default_rng(3).standard_normal((S.grid.npoints, K)).astype(np.float32))
    cbar = to_lta(st, S, O.random_coeffs(So.spectrum, K, seed=4))

    def syn_adj():
        out = st.LowerTriangularArray(torch.zeros(K, S.spectrum.nlm, dtype=torch.complex64, device="cuda"),
                                      S.spectrum)
        st.spec2grid_pullback_(out, gbar, S, unscale_coslat=True)
        return np_of(out)

    def ana_adj():
        out = st.Field(torch.zeros(K, S.grid.npoints, device="cuda"), S.grid)
        st.grid2spec_pullback_(out, cbar, S)
        return np_of(out)

    a, b = _both(S, syn_adj)
    assert _rel(a, b) < MODE_TOL
    a, b = _both(S, ana_adj)
    assert _rel(a, b) < MODE_TOL


@pytest.mark.parametrize("prec", ["fp16x3", "bf16x5"])
def test_t511_tensor_vs_direct(st, prec):
    """T511 x 64 (primes up to 383: two 128-row tiles of the stage matrices)."""
    S, So = setup(st, 511, "octa", 64, precision=prec)
    K = 64
    c = O.random_coeffs(So.spectrum, K, seed=17)
    lta = to_lta(st, S, c)

    def syn():
        f = nan_field(st, S, K)
        st.transform_(f, lta, S)
        return np_of(f)

    ft, fd = _both(S, syn)
    assert np.all(np.isfinite(ft))
    assert _rel(ft, fd) < MODE_TOL
    field = to_field(st, S, ft.astype(np.float32))

    def ana():
        out = nan_lta(st, S, K)
        st.transform_(out, field, S)
        return np_of(out)

    at, ad = _both(S, ana)
    assert np.all(np.isfinite(at))
    assert _rel(at, ad) < MODE_TOL


@pytest.mark.parametrize("K", [1, 3])
def test_strided_views_tensor_vs_direct(st, K):
    """Row views of larger parents (leading dimensions not multiples of 4: the FFT kernel's
    unaligned paths) and one or three layers."""
    import torch
    S, So = setup(st, 127, "octa", 8)
    c = O.random_coeffs(So.spectrum, K, seed=21 + K)
    parent = torch.zeros(K + 2, S.spectrum.nlm + 17, dtype=torch.complex64, device="cuda")
    parent[1:K + 1, :S.spectrum.nlm] = torch.tensor(c.T, dtype=torch.complex64, device="cuda")
    lt = st.LowerTriangularArray(parent[1:K + 1, :S.spectrum.nlm], S.spectrum)
    gparent = torch.full((K + 2, S.grid.npoints + 5), 7.0, device="cuda")

    def syn():
        gparent.fill_(7.0)
        f = st.Field(gparent[1:K + 1, :S.grid.npoints], S.grid)
        st.transform_(f, lt, S)
        assert torch.all(gparent[0] == 7.0) and torch.all(gparent[K + 1] == 7.0)
        assert torch.all(gparent[1:K + 1, S.grid.npoints:] == 7.0)
        return np_of(f)

    ft, fd = _both(S, syn)
    assert _rel(ft, fd) < MODE_TOL
    assert O.rel_err(ft, So.synthesize(c)) < TOL
    gparent.fill_(7.0)
    gparent[1:K + 1, :S.grid.npoints] = torch.tensor(ft.T, dtype=torch.float32, device="cuda")
    field = st.Field(gparent[1:K + 1, :S.grid.npoints], S.grid)

    def ana():
        op = torch.full((K + 2, S.spectrum.nlm + 17), complex("nan+nanj"), dtype=torch.complex64, device="cuda")
        out = st.LowerTriangularArray(op[1:K + 1, :S.spectrum.nlm], S.spectrum)
        st.transform_(out, field, S)
        assert torch.all(torch.isnan(op[0])) and torch.all(torch.isnan(op[1:K + 1, S.spectrum.nlm:]))
        return np_of(out)

    at, ad = _both(S, ana)
    assert np.all(np.isfinite(at))
    assert _rel(at, ad) < MODE_TOL
