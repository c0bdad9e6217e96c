"""Tensor-core (tcgen05) split-precision Legendre stage against the FP64 oracle.

Tolerances (relative L2 vs FP64) at T31-T127, measured per direction (worst of 16
layers, T31-T255): split BF16 with 3 products 5.7e-6 (round trip 7.8e-6), so 1e-5;
the 5-product form (Legendre polynomials in three BF16 pieces) 4.3e-6, so 5e-6;
split FP16 with 3 products (11-bit pieces, power-of-two scaling of the Legendre
polynomials per order and of the data per order and layer or per layer) 5e-7, so 1e-6. The T511 x 64 tests
check each layer against the 1e-5 bar (FP16 and the 5-product BF16 meet it; the
3-product BF16 does not on every layer, and its test pins its level).
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import nan_field, nan_lta, np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 1e-5, "bf16x5": 5e-6, "fp16x3": 1e-6}


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


T511_LAYERS = list(range(0, 64, 9))    # 8 layers spread over the 64 of the benchmark


def _t511(st, prec):
    """T511 x 64 (octahedral, nlat 768) round trip and analysis of a band-limited grid:
    per-layer relative L2 errors vs FP64 on 8 layers spread over the batch."""
    S, So = setup(st, 512, "octa", 64, nh=384, precision=prec)
    c = O.random_coeffs(So.spectrum, 64, seed=2)
    f = st.transform(to_lta(st, S, c), S)
    c2 = st.transform(f, S)
    ref = So.synthesize(c[:, T511_LAYERS])
    g32 = ref.astype(np.float32)
    gin = np.zeros((So.grid.npoints, 64), np.float32)
    gin[:, T511_LAYERS] = g32
    c3 = st.transform(to_field(st, S, gin), S)
    assert S.device_status() == 0
    fs, cs, c3s = np_of(f)[:, T511_LAYERS], np_of(c2)[:, T511_LAYERS], np_of(c3)[:, T511_LAYERS]
    ref_rt, ref_an = So.analyze(ref), So.analyze(g32.astype(np.float64))
    per = lambda x, r: [O.rel_err(x[:, i], r[:, i]) for i in range(len(T511_LAYERS))]   # noqa: E731
    return {"syn": per(fs, ref), "rt": per(cs, ref_rt), "ana": per(c3s, ref_an),
            "syn_all": O.rel_err(fs, ref), "rt_all": O.rel_err(cs, ref_rt)}


@pytest.mark.parametrize("prec", ["fp16x3", "bf16x5"])
def test_tc_t511_every_layer_within_1e5(st, prec):
    """The benchmark's size at the north star's bar: every checked layer's synthesis,
    round trip and analysis within 1e-5 of FP64 (measured worst layers: fp16x3 7.6e-7 /
    2.3e-6 / 1.7e-6, bf16x5 6.6e-6 / 6.5e-6 / 2.3e-6)."""
    e = _t511(st, prec)
    assert max(e["syn"]) <= 1e-5 and max(e["rt"]) <= 1e-5 and max(e["ana"]) <= 1e-5, e


def test_bf16x3_t511_error_level(st):
    """Split BF16 with three products at T511 x 64: the two 8-bit pieces of the Legendre
    polynomials and of the data each leave a residual of up to 2^-18, so the synthesis
    alone is ~5e-6 and the round trip ~1e-5 (FP64 emulation of the split with exact
    accumulation: synthesis 4.6e-6). It does NOT meet 1e-5 on every layer (about a
    quarter of the 64 layers exceed it), so it is not the benchmark's headline form;
    this test pins its level."""
    e = _t511(st, "bf16x3")
    assert e["syn_all"] < 8e-6 and e["rt_all"] < 1.4e-5, e
    assert max(e["syn"]) < 1.5e-5 and max(e["rt"]) < 2.5e-5, e


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
