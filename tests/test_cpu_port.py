"""The oracle's C restatement (CPU baseline) agrees with the FP64 numpy oracle."""
import numpy as np
import pytest

import sht_oracle as O
from sht_cpu import CpuTransform


@pytest.mark.parametrize("kind,T", [(O.FULL_GAUSSIAN, 31), (O.OCTAHEDRAL_GAUSSIAN, 63)])
def test_cpu_port_matches_oracle(kind, T):
    nh = O.get_nlat_half(T)
    So = O.SpectralTransform(O.Spectrum(T, T), O.Grid(kind, nh))
    Cp = CpuTransform(kind, nh, T, T, 4)
    c = O.random_coeffs(So.spectrum, 4, seed=1)
    f = Cp.synthesize(c.T)
    ref = So.synthesize(c)
    assert O.rel_err(f.T, ref) < 1e-5
    a = Cp.analyze(f)
    assert O.rel_err(a.T, So.analyze(f.T.astype(np.float64))) < 1e-5
