"""Fused transforms (FFT and Legendre stage in one launch per direction, thread-block
clusters exchanging the Fourier rows through shared memory) against the separate kernels
and the FP64 oracle.

The fused kernels compute every value with the separate kernels' operations in the same
order, so synthesis and analysis give the same bits (tested with torch.equal), including
odd layer counts, one layer, 48 layers (several clusters), unscale_coslat and add; two
calls give the same bits; both stay within 1e-5 of FP64 (relative L2).
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

CASES = [(31, "full", 24, 8), (31, "octa", 24, 5), (63, "octa", 48, 8), (63, "octa", 48, 1), (127, "octa", 96, 48),
         (63, "full", 48, 13), (127, "full", 96, 8),
         (7, "full", 4, 3), (5, "octa", 3, 11)]       # fewer rings than a cluster has CTAs


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


def _pair(st, S, fn):
    """fn() with fusion off, then on: the two results (the plan's mode restored)."""
    mode = S.fusion
    try:
        S.fusion = False
        a = fn()
        S.fusion = True
        b = fn()
    finally:
        S.fusion = mode
    return a, b


@pytest.mark.parametrize("T,grid,nh,K", CASES)
def test_fused_equals_separate_kernels(st, T, grid, nh, K):
    import torch
    S, So = setup(st, T, grid, K, one_more=True, nh=nh)
    assert S.fusion_available
    c = O.random_coeffs(So.spectrum, K, seed=T + K)
    lt = to_lta(st, S, c)
    f0, f1 = _pair(st, S, lambda: st.transform(lt, S))
    assert torch.equal(f0.data, f1.data)
    f2 = _pair(st, S, lambda: st.transform(lt, S))[1]
    assert torch.equal(f2.data, f1.data)                           # deterministic
    ref = So.synthesize(c)
    assert O.rel_err(np_of(f1), ref) < 1e-5
    g = to_field(st, S, ref.astype(np.float32))
    a0, a1 = _pair(st, S, lambda: st.transform(g, S))
    assert torch.equal(a0.data, a1.data)
    assert S.device_status() == 0
    assert O.rel_err(np_of(a1), So.analyze(ref.astype(np.float32).astype(np.float64))) < 1e-5


def test_fused_flags(st):
    """unscale_coslat on the synthesis and add on both directions, fused vs separate."""
    import torch
    T, nh, K = 63, 48, 8
    S, So = setup(st, T, "octa", K, one_more=True, nh=nh)
    c = O.random_coeffs(So.spectrum, K, seed=7)
    lt = to_lta(st, S, c)
    u0, u1 = _pair(st, S, lambda: st.transform(lt, S, unscale_coslat=True))
    assert torch.equal(u0.data, u1.data)
    assert O.rel_err(np_of(u1), So.synthesize(c, unscale_coslat=True)) < 1e-5
    base_f = st.transform(lt, S)
    base_c = st.transform(base_f, S)

    def add_syn():
        f = st.Field(base_f.data.clone(), S.grid)
        st.transform_(f, lt, S, add=True)
        return f

    def add_ana():
        a = st.LowerTriangularArray(base_c.data.clone(), S.spectrum)
        st.transform_(a, base_f, S, add=True)
        return a
    s0, s1 = _pair(st, S, add_syn)
    assert torch.equal(s0.data, s1.data)
    a0, a1 = _pair(st, S, add_ana)
    assert torch.equal(a0.data, a1.data)
    assert S.device_status() == 0


def test_default_mode(st):
    """Fused by default on the small full grid, separate on octahedral grids."""
    S, _ = setup(st, 31, "full", 8, one_more=True, nh=24)
    assert S.fusion
    S, _ = setup(st, 63, "octa", 8, one_more=True, nh=48)
    assert not S.fusion


def test_fusion_unavailable_for_tensor_core_plans(st):
    from speedytransforms import _lib
    S, _ = setup(st, 63, "octa", 8, nh=48, precision="bf16x3")
    assert not S.fusion_available
    with pytest.raises(_lib.ShtError):
        S.fusion = True
    assert not S.fusion
