"""The allocation-free analysis entry point gives the same coefficients as sht_analyze.

sht_analyze_static_scratch serves callers that cannot call cudaMalloc where they
transform: a host with a fixed memory pool handed out at start-up, or a runtime that
forbids allocating once it is initialised. Its Fourier scratch is a fixed 8 MiB array
inside the library instead of the plan's.

It runs the same two FP32 kernels as sht_analyze on the same inputs, so the tests
expect the same bits. They call it through the C ABI twice in a row on different
inputs (the shared array keeps the first call's contents), with fewer layers than
the plan holds, with SHT_ADD, and compare with the FP64 oracle too. Each test
creates its own plan so that it passes alone in a fresh process and after the other
tests; the file name makes pytest collect it last.
"""
import numpy as np
import pytest

import sht_oracle as O

pytestmark = pytest.mark.gpu

T, NLAYERS = 63, 8


def _plan():
    import speedytransforms as st
    sp = st.Spectrum(T, T)
    grid = st.OctahedralGaussianGrid(st.get_nlat_half(T))
    S = st.SpectralTransform(sp, grid, nlayers=NLAYERS, precision="fp32")
    So = O.SpectralTransform(O.Spectrum(T, T), O.Grid(O.OCTAHEDRAL_GAUSSIAN, grid.nlat_half))
    return S, So


def _both(S, g, K, flags, init=None):
    """(static-scratch result, sht_analyze result) for the first K layers of g."""
    import torch
    from speedytransforms import _lib
    nlm, npts = S.spectrum.nlm, S.grid.npoints
    stream = torch.cuda.current_stream().cuda_stream
    fill = init if init is not None else torch.full((NLAYERS, nlm), float("nan"), dtype=torch.complex64,
                                                     device="cuda")
    ref, out = fill.clone(), fill.clone()
    _lib.check(_lib.lib.sht_analyze(S.handle, g.data_ptr(), npts, ref.data_ptr(), nlm, K, flags, stream))
    _lib.check(_lib.lib.sht_analyze_static_scratch(S.handle, g.data_ptr(), npts, out.data_ptr(), nlm, K, flags,
                                                   stream))
    torch.cuda.synchronize()
    return out.cpu().numpy(), ref.cpu().numpy()


def test_static_scratch_analysis_matches_sht_analyze():
    import torch
    S, So = _plan()
    for seed, K in ((5, NLAYERS), (6, NLAYERS), (7, 3)):    # calls in a row; the last with K < nlayers
        c = O.random_coeffs(So.spectrum, NLAYERS, seed=seed)
        gd = So.synthesize(c)
        g = torch.tensor(np.ascontiguousarray(gd.T), dtype=torch.float32, device="cuda")
        a, b = _both(S, g, K, 0)
        assert np.all(np.isfinite(a[:K]))
        assert np.array_equal(a[:K].view(np.uint64), b[:K].view(np.uint64))   # same kernels: same bits
        assert np.all(np.isnan(a[K:]))                                        # layers past K untouched
        ref = So.analyze(gd.astype(np.float32).astype(np.float64)[:, :K])
        assert O.rel_err(a[:K].T.astype(np.complex128), ref) < 1e-5


def test_static_scratch_analysis_add():
    import torch
    from speedytransforms import _lib
    S, So = _plan()
    c = O.random_coeffs(So.spectrum, NLAYERS, seed=8)
    g = torch.tensor(np.ascontiguousarray(So.synthesize(c).T), dtype=torch.float32, device="cuda")
    init = torch.tensor(np.ascontiguousarray(c.T), dtype=torch.complex64, device="cuda")
    a, b = _both(S, g, NLAYERS, _lib.ADD, init=init)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    np.testing.assert_allclose(a, 2 * init.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_static_scratch_rejects_oversized_calls():
    import torch
    import speedytransforms as st
    from speedytransforms import _lib
    sp = st.Spectrum(512, 512)
    grid = st.OctahedralGaussianGrid(384)
    K = 64
    S = st.SpectralTransform(sp, grid, nlayers=K, precision="fp32")
    # real buffers of the call's full size, so that nothing could be out of bounds even if
    # the size check were moved behind a launch
    g = torch.zeros((K, grid.npoints), dtype=torch.float32, device="cuda")
    out = torch.zeros((K, sp.nlm), dtype=torch.complex64, device="cuda")
    rc = _lib.lib.sht_analyze_static_scratch(S.handle, g.data_ptr(), grid.npoints, out.data_ptr(), sp.nlm, K, 0,
                                             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == _lib.SHT_EINVAL
    assert b"8 MiB" in _lib.lib.sht_last_error()
    assert not out.any()
