"""Adjoint transforms (sht_synthesize_adjoint / sht_analyze_adjoint) against the FP64
oracle's restatement of the reference's pullbacks (SpeedyTransformsEnzymeExt.jl:263-323),
which tests/test_oracle.py pins as the exact adjoints by dot products.
Tolerances (relative L2): FP32 1e-5; split BF16 x3 3e-5; split FP16 x3 5e-6."""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import nan_field, nan_lta, np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "bf16x3": 3e-5, "fp16x3": 5e-6}


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "fp16x3"])
@pytest.mark.parametrize("T,grid,K", [(63, "octa", 4), (31, "full", 3)])
@pytest.mark.parametrize("unscale", [False, True])
def test_synthesis_adjoint(st, prec, T, grid, K, unscale):
    S, So = setup(st, T, grid, K, precision=prec)
    rng = np.random.default_rng(T + K)
    g = rng.standard_normal((So.grid.npoints, K)).astype(np.float32)
    out = nan_lta(st, S, K)
    st.spec2grid_pullback_(out, to_field(st, S, g), S, unscale_coslat=unscale, add=False)
    assert S.device_status() == 0
    ref = So.synthesize_adjoint(g.astype(np.float64), unscale_coslat=unscale)
    assert O.rel_err(np_of(out), ref) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "fp16x3"])
@pytest.mark.parametrize("T,grid,K", [(63, "octa", 4), (31, "full", 3)])
def test_analysis_adjoint(st, prec, T, grid, K):
    S, So = setup(st, T, grid, K, precision=prec)
    c = O.random_coeffs(So.spectrum, K, seed=T)
    out = nan_field(st, S, K)
    st.grid2spec_pullback_(out, to_lta(st, S, c), S, add=False)
    assert S.device_status() == 0
    assert O.rel_err(np_of(out), So.analyze_adjoint(c)) < TOL[prec]


def test_adjoints_accumulate_and_dot_products(st):
    """add (the reference's accumulate) and the adjoint identities on the GPU results."""
    import torch
    S, So = setup(st, 63, "octa", 4, precision="fp32")
    rng = np.random.default_rng(1)
    c = O.random_coeffs(So.spectrum, 4, seed=3)
    g = rng.standard_normal((So.grid.npoints, 4)).astype(np.float32)
    # accumulate: outputs = prefilled + adjoint, compared as sums (FP32 rounding of the sum)
    cbar = st.spec2grid_pullback_(to_lta(st, S, c), to_field(st, S, g), S)
    gbar = st.grid2spec_pullback_(to_field(st, S, g), to_lta(st, S, c), S)
    torch.cuda.synchronize()
    assert O.rel_err(np_of(cbar), c + So.synthesize_adjoint(g.astype(np.float64))) < 1e-6
    assert O.rel_err(np_of(gbar), g + So.analyze_adjoint(c)) < 1e-6
    # <S c, g> = <c, S^T g> and <A g, c> = <g, A^T c> on the GPU results
    f = np_of(st.transform(to_lta(st, S, c), S)).astype(np.float64)
    st_g = np_of(st.spec2grid_pullback_(nan_lta(st, S, 4), to_field(st, S, g), S, add=False))
    a = np_of(st.transform(to_field(st, S, g), S))
    at_c = np_of(st.grid2spec_pullback_(nan_field(st, S, 4), to_lta(st, S, c), S, add=False)).astype(np.float64)
    lhs, rhs = float(np.sum(f * g)), float(np.sum(c.real * st_g.real) + np.sum(c.imag * st_g.imag))
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)
    lhs, rhs = float(np.sum(a.real * c.real) + np.sum(a.imag * c.imag)), float(np.sum(g * at_c))
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)
