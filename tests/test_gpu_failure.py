"""Failure detection of the tensor-core kernels' bounded waits, without a GPU fault: a wait
on an mbarrier phase that nothing completes gives up after its limit, its code reaches the
plan's status word, and the context keeps computing the same bits afterwards."""
import time

import numpy as np
import pytest
import torch

import speedytransforms as st
import speedytransforms._lib as L
import sht_oracle as O

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def round_trip(S, spec, grid, coeffs):
    f = st.Field.zeros(grid, coeffs.shape[0], device=DEV)
    out = st.LowerTriangularArray.zeros(spec, coeffs.shape[0], device=DEV)
    st.transform_(f, st.LowerTriangularArray(coeffs, spec), S)
    st.transform_(out, f, S)
    torch.cuda.synchronize()
    return f.data.clone(), out.data.clone()


@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_expired_wait_reports_and_context_survives(precision):
    K = 8
    spec, grid = st.Spectrum(64, 64), st.OctahedralGaussianGrid(48)
    S = st.SpectralTransform(spec, grid, nlayers=K, precision=precision, device=DEV)
    c = O.random_coeffs(O.Spectrum(64, 64), K, seed=11)
    coeffs = torch.tensor(np.ascontiguousarray(c.T), dtype=torch.complex64).to(DEV)
    before = round_trip(S, spec, grid, coeffs)
    assert S.device_status() == 0

    t0 = time.perf_counter()
    S.diag_wait_expiry(20000)                     # 20 ms limit
    status = S.device_status()                    # synchronises
    dt = time.perf_counter() - t0
    assert status == L.SHT_STATUS_DIAG_EXPIRED
    assert 0.02 <= dt < 5.0
    assert S.device_status() == 0                 # reading the word clears it

    after = round_trip(S, spec, grid, coeffs)     # the context is still usable
    assert torch.equal(before[0], after[0]) and torch.equal(before[1], after[1])
    assert S.device_status() == 0


def test_limit_is_checked():
    S = st.SpectralTransform(st.Spectrum(32, 32), st.OctahedralGaussianGrid(24), nlayers=1, device=DEV)
    for bad in (0, -5, 1000001):
        with pytest.raises(Exception):
            S.diag_wait_expiry(bad)
    assert S.device_status() == 0
