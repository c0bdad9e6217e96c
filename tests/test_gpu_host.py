"""Transforms with coefficients in host memory (sht_synthesize_host / sht_analyze_host):
the chunked, copy-overlapped path gives the device path's results bit for bit, for ragged
chunks, padded leading dimensions, page-locked and pageable buffers, and per-chunk round
trips whose copies overlap one another."""
import numpy as np
import pytest
import torch

import speedytransforms as st
import sht_oracle as O

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def setup(T, nh, K, precision="fp32", chunk=None):
    spec = st.Spectrum(T + 1, T + 1)
    grid = st.OctahedralGaussianGrid(nh)
    S = st.SpectralTransform(spec, grid, nlayers=K, precision=precision, device=DEV)
    if chunk is not None:
        S.set_host_chunk(chunk)
    c = O.random_coeffs(O.Spectrum(T + 1, T + 1), K, seed=T + K)
    coeffs = torch.tensor(np.ascontiguousarray(c.T), dtype=torch.complex64)
    return S, spec, grid, coeffs


@pytest.mark.parametrize("precision", ["fp32", "bf16x3", "fp16x3", "bf16x5"])
def test_synthesize_analyze_host_match_device(precision):
    K = 20
    S, spec, grid, coeffs = setup(63, 48, K, precision, chunk=8)      # chunks 8, 8, 4
    pad = spec.nlm + 5
    host = torch.zeros((K, pad), dtype=torch.complex64).pin_memory()
    host[:, :spec.nlm] = coeffs
    lt_host = st.LowerTriangularArray(host[:, :spec.nlm], spec)            # ldc = nlm + 5
    lt_dev = st.LowerTriangularArray(coeffs.to(DEV), spec)
    f_host = st.Field.zeros(grid, K, device=DEV)
    f_dev = st.Field.zeros(grid, K, device=DEV)
    st.transform_(f_host, lt_host, S)
    st.transform_(f_dev, lt_dev, S)
    torch.cuda.synchronize()
    assert torch.equal(f_host.data, f_dev.data)

    out_host = torch.full((K, pad), complex(np.nan, np.nan), dtype=torch.complex64).pin_memory()
    out_dev = st.LowerTriangularArray.zeros(spec, K, device=DEV)
    st.transform_(st.LowerTriangularArray(out_host[:, :spec.nlm], spec), f_dev, S)
    st.transform_(out_dev, f_dev, S)
    S.host_wait()
    torch.cuda.synchronize()
    assert torch.equal(out_host[:, :spec.nlm], out_dev.data.cpu())
    assert torch.isnan(out_host[:, spec.nlm:].real).all()                 # the padding is untouched
    assert S.device_status() == 0


def test_chunked_round_trips_overlap():
    """Round trips issued chunk by chunk (synthesis then analysis of each chunk), so the
    copy in of chunk i + 1 and the copy out of chunk i - 1 overlap the work of chunk i."""
    K, ch = 32, 8
    S, spec, grid, coeffs = setup(127, 96, K, "bf16x3", chunk=ch)
    host_in = coeffs.pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    field = st.Field.zeros(grid, K, device=DEV)
    for rep in range(2):
        host_out.zero_()
        for k0 in range(0, K, ch):
            f = st.Field(field.data[k0:k0 + ch], grid)
            st.transform_(f, st.LowerTriangularArray(host_in[k0:k0 + ch], spec), S)
            st.transform_(st.LowerTriangularArray(host_out[k0:k0 + ch], spec), f, S)
        S.host_wait()
        torch.cuda.synchronize()
        ref_f = st.Field.zeros(grid, K, device=DEV)
        ref = st.LowerTriangularArray.zeros(spec, K, device=DEV)
        st.transform_(ref_f, st.LowerTriangularArray(coeffs.to(DEV), spec), S)
        st.transform_(ref, ref_f, S)
        torch.cuda.synchronize()
        assert torch.equal(host_out, ref.data.cpu())
        # the round trip reproduces the band-limited input (spectral_transform.jl round-trip
        # tests) to the split-BF16 accuracy (relative L2 1.0e-5 at T127)
        err = torch.linalg.norm(host_out - coeffs) / torch.linalg.norm(coeffs)
        assert err < 2e-5


def test_pageable_host_memory_and_errors():
    K = 6
    S, spec, grid, coeffs = setup(31, 24, K)
    f = st.Field.zeros(grid, K, device=DEV)
    st.transform_(f, st.LowerTriangularArray(coeffs.clone(), spec), S)     # pageable
    ref = st.Field.zeros(grid, K, device=DEV)
    st.transform_(ref, st.LowerTriangularArray(coeffs.to(DEV), spec), S)
    torch.cuda.synchronize()
    assert torch.equal(f.data, ref.data)
    out = st.LowerTriangularArray(torch.zeros((K, spec.nlm), dtype=torch.complex64), spec)
    with pytest.raises(TypeError):
        st.transform_(out, f, S, add=True)
    with pytest.raises(st.DimensionMismatch):
        st.transform_(st.Field.zeros(grid, K + 1, device=DEV),
                      st.LowerTriangularArray(torch.zeros((K + 1, spec.nlm), dtype=torch.complex64), spec), S)
