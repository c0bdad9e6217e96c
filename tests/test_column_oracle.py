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
