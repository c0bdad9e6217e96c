"""Tensor-core (tcgen05) split-precision Legendre stage against the FP64 oracle.

Tolerances (relative L2 vs FP64): split BF16 with 3 products keeps ~16 bits of each
operand, so 3e-5 per direction; the 5-product form (Legendre polynomials in three
BF16 pieces) 1e-5; split FP16 with 3 products (~22 bits, power-of-two scaling of
the Legendre polynomials per order and of the data per layer) 5e-6: the split itself
is below 1e-6, the rest is the tensor core's FP32 accumulation and the cancellation
of the Legendre sums (a T511 round trip measures ~3e-6).
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import nan_field, nan_lta, np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 3e-5, "bf16x5": 1e-5, "fp16x3": 5e-6}


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


@pytest.mark.parametrize("prec", ["bf16x3", "bf16x5", "fp16x3"])
@pytest.mark.parametrize("T,grid,K", [(63, "octa", 8), (31, "full", 4), (127, "octa", 48)])
def test_tc_synthesis_analysis(st, prec, T, grid, K):
    S, So = setup(st, T, grid, K, precision=prec)
    c = O.random_coeffs(So.spectrum, K, seed=T + 3)
    f = nan_field(st, S, K)
    st.transform_(f, to_lta(st, S, c), S)
    assert S.device_status() == 0
    got = np_of(f)
    assert np.all(np.isfinite(got))
    assert O.rel_err(got, So.synthesize(c)) < TOL[prec]
    g = So.synthesize(c).astype(np.float32)
    out = nan_lta(st, S, K)
    st.transform_(out, to_field(st, S, g), S)
    assert S.device_status() == 0
    a = np_of(out)
    assert np.all(np.isfinite(a))
    assert O.rel_err(a, So.analyze(g.astype(np.float64))) < TOL[prec]


@pytest.mark.parametrize("prec", ["bf16x3", "bf16x5", "fp16x3"])
def test_tc_odd_layers_and_add(st, prec):
    import torch
    S, So = setup(st, 63, "octa", 8, precision=prec)
    c = O.random_coeffs(So.spectrum, 5, seed=1)
    f = st.transform(to_lta(st, S, c), S)
    assert O.rel_err(np_of(f), So.synthesize(c)) < TOL[prec]
    out = st.transform(f, S)
    acc = st.LowerTriangularArray(out.data.clone(), S.spectrum)
    st.transform_(acc, f, S, add=True)
    assert S.device_status() == 0
    np.testing.assert_allclose(np_of(acc), 2 * np_of(out), rtol=1e-6, atol=1e-7)
    del torch


def test_tc_t511_full_size(st):
    S, So = setup(st, 512, "octa", 64, nh=384, precision="bf16x5")
    c = O.random_coeffs(So.spectrum, 64, seed=2)
    f = st.transform(to_lta(st, S, c), S)
    c2 = st.transform(f, S)
    assert S.device_status() == 0
    sub = [0, 63]
    ref = So.synthesize(c[:, sub])
    assert O.rel_err(np_of(f)[:, sub], ref) < 1e-5
    assert O.rel_err(np_of(c2)[:, sub], So.analyze(ref)) < 1e-5


@pytest.mark.parametrize("scale", [1e4, 1e-4])
def test_fp16x3_data_scaling(st, scale):
    """Layers far outside fp16's range (x 1e4, x 1e-4) and an all-zero layer: the
    per-layer power-of-two data scaling keeps the split-FP16 error at its usual level."""
    S, So = setup(st, 63, "octa", 8, precision="fp16x3")
    c = O.random_coeffs(So.spectrum, 4, seed=5) * scale
    c[:, 2] = 0.0
    f = st.transform(to_lta(st, S, c), S)
    assert S.device_status() == 0
    got = np_of(f)
    assert np.all(got[:, 2] == 0.0)
    ref = So.synthesize(c)
    assert O.rel_err(got, ref) < TOL["fp16x3"]
    out = st.transform(to_field(st, S, ref.astype(np.float32)), S)
    a = np_of(out)
    assert np.all(a[:, 2] == 0.0)
    assert O.rel_err(a, So.analyze(ref.astype(np.float32).astype(np.float64))) < TOL["fp16x3"]


def test_fp16x3_t511_full_size(st):
    S, So = setup(st, 512, "octa", 64, nh=384, precision="fp16x3")
    c = O.random_coeffs(So.spectrum, 64, seed=2)
    f = st.transform(to_lta(st, S, c), S)
    c2 = st.transform(f, S)
    assert S.device_status() == 0
    sub = [0, 63]
    ref = So.synthesize(c[:, sub])
    assert O.rel_err(np_of(f)[:, sub], ref) < TOL["fp16x3"]
    assert O.rel_err(np_of(c2)[:, sub], So.analyze(ref)) < TOL["fp16x3"]
