"""One time step's transforms of the primitive-equation wet model (T63, 8 layers), in the
reference's order (SpeedyWeather/src/time_stepping/transform.jl:117-191,
SpeedyWeather/src/dynamics/tendencies.jl:161-214, 585-594):

* every output of the sequence (prognostic and velocity grids, the surface-pressure
  gradient grid, the analysed grid tendencies and the spectral tendencies the operators
  accumulate) against the FP64 oracle run through the same sequence;
* the fused form (two one-launch operator sets) equals the separate calls bit for bit;
* captured as one CUDA graph and replayed, the results equal the eager calls bit for bit.

Tolerance (relative L2 per output vs FP64): 1e-5 for the FP32 and the split-FP16 plans.
"""
import numpy as np
import pytest

import sht_oracle as O

pytestmark = pytest.mark.gpu

T, NH, L = 63, 48, 8


def _outs(step):
    return [step.grid_prog.data, step.uv_grid.data, step.dpres_grid.data, step.spec_tend.data, step.tend.data]


def _oracle(step):
    """The step's sequence in FP64 on the step's own inputs (prognostic coefficients and
    grid tendencies): the same calls as DycoreStep.__call__, restated with the oracle."""
    sp = O.Spectrum(T + 2, T + 1)
    So = O.SpectralTransform(sp, O.Grid(O.OCTAHEDRAL_GAUSSIAN, NH))
    P = step.prog.data.cpu().numpy().T.astype(np.complex128)             # [nlm, 4L + 1]
    G = step.grid_tend.data.cpu().numpy().T.astype(np.float64)            # [npoints, 9L + 1]
    dpdx, dpdy = O.gradient(sp, P[:, 4 * L])
    dpres_grid = So.synthesize(np.stack([dpdx, dpdy], axis=1), unscale_coslat=True)
    U, V = O.UV_from_vordiv(sp, P[:, 0:L], P[:, L:2 * L])
    grid_prog = So.synthesize(P)
    uv_grid = So.synthesize(np.concatenate([U, V], axis=1), unscale_coslat=True)
    Tn = So.analyze(G)
    u, v = Tn[:, 0:L], Tn[:, L:2 * L]
    z = np.zeros((sp.nlm, L), np.complex128)
    vor_t = O.curl(sp, u, v, add=True, out=z)
    div_t = O.divergence(sp, u, v, add=True, out=z)
    temp_t = O.divergence(sp, Tn[:, 3 * L + 1:4 * L + 1], Tn[:, 4 * L + 1:5 * L + 1], add=True, flipsign=True, out=z)
    hum_t = O.divergence(sp, Tn[:, 7 * L + 1:8 * L + 1], Tn[:, 8 * L + 1:9 * L + 1], add=True, flipsign=True, out=z)
    div_t = O.laplace(sp, Tn[:, 5 * L + 1:6 * L + 1], add=True, flipsign=True, out=div_t)
    tend = np.concatenate([vor_t, div_t, temp_t, hum_t], axis=1)
    return [grid_prog, uv_grid, dpres_grid, Tn, tend]


@pytest.mark.parametrize("precision", ["fp32", "fp16x3"])
def test_step_matches_oracle(precision):
    import torch
    import speedytransforms as st
    step = st.DycoreStep(T=T, nlat_half=NH, L=L, precision=precision)
    step()
    torch.cuda.synchronize()
    assert step.S.device_status() == 0
    names = ["grid_prog", "uv_grid", "dpres_grid", "spec_tend", "tend"]
    for name, got, ref in zip(names, _outs(step), _oracle(step)):
        g = got.cpu().numpy().T
        g = g.astype(np.complex128 if np.iscomplexobj(g) else np.float64)
        assert np.all(np.isfinite(g)), name
        assert O.rel_err(g, ref) < 1e-5, (name, O.rel_err(g, ref))


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_fused_equals_separate_calls(precision):
    import torch
    import speedytransforms as st
    a = st.DycoreStep(T=T, nlat_half=NH, L=L, precision=precision, fused=True)
    b = st.DycoreStep(T=T, nlat_half=NH, L=L, precision=precision, fused=False)
    a()
    b()
    torch.cuda.synchronize()
    assert a.launches() == 7 and b.launches() == 11
    for x, y in zip(_outs(a), _outs(b)):
        assert torch.equal(x, y)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_graph_replay_equals_eager(precision):
    import torch
    import speedytransforms as st
    step = st.DycoreStep(T=T, nlat_half=NH, L=L, precision=precision)
    step()
    torch.cuda.synchronize()
    eager = [o.clone() for o in _outs(step)]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        step()
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    for o in _outs(step):
        o.zero_()
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(_outs(step), eager):
        assert torch.equal(a, b)
    graph.replay()                          # replays again (the step resets its accumulators)
    torch.cuda.synchronize()
    for a, b in zip(_outs(step), eager):
        assert torch.equal(a, b)
    assert step.S.device_status() == 0
