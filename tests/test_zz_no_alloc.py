"""The allocation-free analysis entry point gives the same coefficients as sht_analyze.

sht_analyze_static_scratch serves callers that cannot call cudaMalloc where they
transform (inside a CUDA-graph capture they do not own, under a fixed memory pool
set up at start, or in a runtime that forbids allocating after initialisation):
its Fourier scratch is a fixed 8 MiB array inside the library. The test calls it
through the C ABI twice in a row, on different inputs, and compares each result
with sht_analyze on the same plan (same FP32 kernels, so within 1e-6 relative).
It creates its own plan so it passes alone in a fresh process and after the other
tests; the file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

import sht_oracle as O

pytestmark = pytest.mark.gpu


def test_static_scratch_analysis_matches_sht_analyze():
    import torch

    import speedytransforms as st
    from speedytransforms import _lib

    T, K = 63, 8
    sp = st.Spectrum(T, T)
    grid = st.OctahedralGaussianGrid(st.get_nlat_half(T))
    S = st.SpectralTransform(sp, grid, nlayers=K, precision="fp32")
    So = O.SpectralTransform(O.Spectrum(T, T), O.Grid(O.OCTAHEDRAL_GAUSSIAN, grid.nlat_half))
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (5, 6):                    # two calls in a row on different inputs
        c = O.random_coeffs(So.spectrum, K, seed=seed)
        g = torch.tensor(np.ascontiguousarray(So.synthesize(c).T), dtype=torch.float32, device="cuda")
        ref = torch.full((K, sp.nlm), float("nan"), dtype=torch.complex64, device="cuda")
        out = torch.full((K, sp.nlm), float("nan"), dtype=torch.complex64, device="cuda")
        _lib.check(_lib.lib.sht_analyze(S.handle, g.data_ptr(), grid.npoints, ref.data_ptr(), sp.nlm, K, 0, stream))
        _lib.check(_lib.lib.sht_analyze_static_scratch(S.handle, g.data_ptr(), grid.npoints, out.data_ptr(), sp.nlm,
                                                       K, 0, stream))
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-6


def test_static_scratch_rejects_oversized_calls():
    import speedytransforms as st
    from speedytransforms import _lib

    sp = st.Spectrum(512, 512)
    grid = st.OctahedralGaussianGrid(384)
    S = st.SpectralTransform(sp, grid, nlayers=64, precision="fp32")
    rc = _lib.lib.sht_analyze_static_scratch(S.handle, ctypes.c_void_p(16), grid.npoints, ctypes.c_void_p(16), sp.nlm,
                                             64, 0, None)
    assert rc == _lib.SHT_EINVAL
    assert b"8 MiB" in _lib.lib.sht_last_error()
