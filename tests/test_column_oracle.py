"""Column-physics oracle (oracle/column_oracle.py) against properties of the schemes it
restates: latent-heat balance of condensation (large_scale_condensation.jl:131-158),
enthalpy conservation of deep and moisture/heat conservation of shallow Betts-Miller
convection (convection.jl:90-130; Frierson 2007 eqs. 5, 11-15), dry columns inert."""
import numpy as np

import column_oracle as C


def test_condensation_latent_heat_balance():
    """A condensing layer at or above the freezing threshold makes no snow (the melting
    heat only enters the implicit correction), so it heats by exactly the latent heat of
    the water it removes: c_p dT = -L_v dq."""
    T, q, u, v, ps = C.synthetic_columns(4000, seed=3)
    dT, dq = C.condensation(T, q, ps)
    sel = (np.abs(dq) > 0) & (T >= C.FREEZING)
    assert sel.sum() > 20
    np.testing.assert_allclose(C.CP * dT[sel], -C.LV * dq[sel], rtol=1e-9)


def test_convection_conservation():
    T, q, u, v, ps = C.synthetic_columns(3000, seed=5)
    dT, dq = C.convection(T, q, ps)
    _, _, dsig = C.sigma_levels()
    heat = (C.CP * dT + C.LV * dq) @ dsig          # column enthalpy tendency
    moist = dq @ dsig
    dry_heat = dT @ dsig
    deep = moist < -1e-15                          # deep convection precipitates (dries)
    assert deep.sum() > 50
    scale = np.abs(C.CP * dT) @ dsig + 1e-30
    assert np.max(np.abs(heat[deep]) / scale[deep]) < 1e-9
    shallow = (np.abs(moist) <= 1e-15 * (np.abs(dq) @ dsig + 1e-30)) & (np.abs(dT).sum(1) > 0)
    assert np.max(np.abs(dry_heat[shallow]) / (np.abs(dT[shallow]) @ dsig)) < 1e-9


def test_dry_columns_do_not_condense():
    T, q, u, v, ps = C.synthetic_columns(500, seed=7)
    dT, dq = C.condensation(T, q * 1e-3, ps)
    assert np.all(dT == 0) and np.all(dq == 0)


def test_float32_mode_tracks_float64():
    T, q, u, v, ps = C.synthetic_columns(500, seed=9)
    a = C.column_tendencies(T, q, ps)
    b = C.column_tendencies(T, q, ps, dtype=np.float32)
    for x, y in zip(a, b):
        same = np.all(np.isclose(x, y, rtol=1e-3, atol=1e-3 * np.abs(x).max()), axis=1)
        assert same.mean() > 0.99


def _random_params(seed):
    rng = np.random.default_rng(seed)
    shapes = [(256, 64), (256, 256), (256, 256), (16, 256)]
    params = []
    for i, (o, n) in enumerate(shapes):
        w = rng.normal(0, np.sqrt(2.0 / n), (o, n))
        if i == 0:
            w[:, 33:] = 0.0
        params.append((w, rng.normal(0, 0.1, o)))
    return params


def test_mlp_backward_finite_differences():
    """The FP64 restatement of the emulator's backward pass against central differences
    of its own loss on a few entries of every layer's weights and biases."""
    rng = np.random.default_rng(7)
    params = _random_params(1)
    xn = rng.normal(size=(48, 33))
    yn = rng.normal(size=(48, 16))
    _, grads = C.mlp_backward(params, xn, yn, bf16=False)
    h = 1e-6
    for layer in range(4):
        w, b = params[layer]
        for _ in range(4):
            i, j = rng.integers(w.shape[0]), rng.integers(33 if layer == 0 else w.shape[1])
            for arr, g in ((w, grads[layer][0][i, j]), (b, grads[layer][1][i])):
                idx = (i, j) if arr.ndim == 2 else (i,)
                old = arr[idx]
                arr[idx] = old + h
                lp = C.mlp_backward(params, xn, yn, bf16=False)[0]
                arr[idx] = old - h
                lm = C.mlp_backward(params, xn, yn, bf16=False)[0]
                arr[idx] = old
                fd = (lp - lm) / (2 * h)
                assert abs(fd - g) <= 1e-6 * max(1e-3, abs(g)) + 1e-9, (layer, idx, fd, g)


def test_bf16_round():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.1415926, 65504.0, 1e-30], np.float32)
    r = C.bf16_round(a)
    import torch
    ref = torch.tensor(a).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(r, ref.astype(np.float64))
    # BF16 rounding of the forward pass stays close to the exact one
    params = _random_params(2)
    xn = np.random.default_rng(3).normal(size=(32, 33))
    y1, _ = C.mlp_forward(params, xn, bf16=True)
    y0, _ = C.mlp_forward(params, xn, bf16=False)
    assert np.linalg.norm(y1 - y0) / np.linalg.norm(y0) < 3e-2
