"""MatrixSpectralTransform (sht_matrix_*): the transforms as dense products.

The matrices are this library's FP32 transforms of unit vectors (matrix_transform.jl:134-173).
The FP32 form computes its products as three TF32 products on the tensor cores (the
matrix split into TF32 pieces in shared memory, the leading product drained every 128
deep into FP32 registers with rounding to nearest), so it agrees with the
SpectralTransform to FP32 rounding; the split 16-bit forms carry their split error.
Against the FP64 oracle: FP32 1e-5; every split 16-bit form 3e-5 (relative L2: one dot
product of length npoints or 2 nlm whose terms cancel heavily, accumulated in 512-deep
chunks in the tensor core's truncating FP32).
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import nan_field, nan_lta, np_of, setup, to_field, to_lta

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "bf16x3": 3e-5, "bf16x5": 3e-5, "fp16x3": 3e-5}
_cache = {}


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


def matrix(st, T, grid, nh, K, prec):
    key = (T, grid, nh, K, prec)
    if key not in _cache:
        g = st.OctahedralGaussianGrid(nh) if grid == "octa" else st.FullGaussianGrid(nh)
        _cache[key] = st.MatrixSpectralTransform(st.Spectrum(T, T), g, nlayers=K, precision=prec)
    return _cache[key]


@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "fp16x3", "bf16x5"])
@pytest.mark.parametrize("T,grid,nh,K", [(31, "full", 24, 3), (63, "octa", 48, 8)])
def test_matrix_transform_vs_oracle(st, prec, T, grid, nh, K):
    M = matrix(st, T, grid, nh, K, prec)
    S, So = setup(st, T, grid, K, nh=nh)
    c = O.random_coeffs(So.spectrum, K, seed=T + 11)
    f = nan_field(st, S, K)
    st.transform_(f, to_lta(st, S, c), M)
    assert M.device_status() == 0
    ref = So.synthesize(c)
    assert O.rel_err(np_of(f), ref) < TOL[prec]
    g = ref.astype(np.float32)
    a = nan_lta(st, S, K)
    st.transform_(a, to_field(st, S, g), M)
    assert M.device_status() == 0
    assert O.rel_err(np_of(a), So.analyze(g.astype(np.float64))) < TOL[prec]


def test_matrix_fp32_matches_spectral_transform(st):
    M = matrix(st, 31, "full", 24, 3, "fp32")
    S, So = setup(st, 31, "full", 3, nh=24)
    c = O.random_coeffs(So.spectrum, 3, seed=4)
    lt = to_lta(st, S, c)
    fm, fs = st.transform(lt, M, unscale_coslat=True), st.transform(lt, S, unscale_coslat=True)
    assert O.rel_err(np_of(fm), np_of(fs)) < 2e-6
    am, as_ = st.transform(fs, M), st.transform(fs, S)
    assert O.rel_err(np_of(am), np_of(as_)) < 2e-6


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
def test_matrix_unscale_and_single_layer(st, prec):
    M = matrix(st, 63, "octa", 48, 8, prec)
    S, So = setup(st, 63, "octa", 8, nh=48)
    c = O.random_coeffs(So.spectrum, 1, seed=9)
    f = st.transform(to_lta(st, S, c), M, unscale_coslat=True)
    ref = So.synthesize(c, unscale_coslat=True)
    assert O.rel_err(np_of(f), ref) < TOL[prec]
    with pytest.raises(TypeError):
        st.transform_(st.Field.zeros(S.grid, 1), to_lta(st, S, c), M, add=True)


def test_matrix_fp32_layer_tiles_and_determinism(st):
    """70 layers (two column tiles of 64) against the oracle; a second call gives the same
    bits; a 5-layer call gives the bits of the first 5 layers of the 70-layer call (each
    layer's sums run in the same fixed order whatever K)."""
    import torch
    M = matrix(st, 31, "full", 24, 70, "fp32")
    S, So = setup(st, 31, "full", 70, nh=24)
    c = O.random_coeffs(So.spectrum, 70, seed=21)
    lt = to_lta(st, S, c)
    f1, f2 = st.transform(lt, M), st.transform(lt, M)
    assert M.device_status() == 0
    assert torch.equal(f1.data, f2.data)
    ref = So.synthesize(c)
    assert O.rel_err(np_of(f1), ref) < TOL["fp32"]
    f5 = st.transform(st.LowerTriangularArray(lt.data[:5].contiguous(), S.spectrum), M)
    assert torch.equal(f5.data, f1.data[:5])
    g = ref.astype(np.float32)
    a1, a2 = st.transform(to_field(st, S, g), M), st.transform(to_field(st, S, g), M)
    assert M.device_status() == 0
    assert torch.equal(a1.data, a2.data)
    assert O.rel_err(np_of(a1), So.analyze(g.astype(np.float64))) < TOL["fp32"]


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
def test_matrix_smaller_than_one_tile(st, prec):
    """T5 on the full grid with nlat 8: matrices of 2 nlm = 42 x npoints = 128, less than one
    128 x 32 tile in one direction and one k-block deep in the other."""
    M = matrix(st, 5, "full", 4, 3, prec)
    S, So = setup(st, 5, "full", 3, nh=4)
    c = O.random_coeffs(So.spectrum, 3, seed=12)
    f = st.transform(to_lta(st, S, c), M)
    assert M.device_status() == 0
    ref = So.synthesize(c)
    assert O.rel_err(np_of(f), ref) < TOL[prec]
    a = st.transform(to_field(st, S, ref.astype(np.float32)), M)
    assert O.rel_err(np_of(a), So.analyze(ref.astype(np.float32).astype(np.float64))) < TOL[prec]
