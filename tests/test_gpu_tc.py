"""Tensor-core (tcgen05) split-precision Legendre stage against the FP64 oracle.

Tolerances (relative L2 vs FP64): split BF16 with 3 products keeps ~16 bits of each
operand, so 3e-5 per direction; the 5-product form (Legendre polynomials in three
BF16 pieces) 1e-5.
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import nan_field, nan_lta, np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 3e-5, "bf16x5": 1e-5}


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


@pytest.mark.parametrize("prec", ["bf16x3", "bf16x5"])
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


@pytest.mark.parametrize("prec", ["bf16x3", "bf16x5"])
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
