"""Batches (sht_batch_*): a mixed batch of transforms in one grouped launch per stage.

The mixed-truncation workload of the batching configuration: octahedral T31 (nlat 48),
T63 (96), T127 (192) and T255 (384) with 1, 8, 16 and 64 layers, FP32, each
synthesised and analysed. The grouped kernels run the same tile bodies in the same
arithmetic order as the per-plan kernels, so the batch's outputs must equal one
transform_ call per item bit for bit; the oracle pins them within the FP32 tolerance.
"""
import numpy as np
import pytest

import sht_oracle as O
from test_gpu_parity import np_of, to_lta

pytestmark = pytest.mark.gpu

MIX = [(32, 24, 1), (64, 48, 8), (128, 96, 16), (256, 192, 64)]   # (T + 1, nlat_half, layers)


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


@pytest.fixture(scope="module")
def mixed(st):
    """Plans, seeded inputs, and the per-call reference outputs of the mixed batch."""
    import torch
    cases = []
    for T, nh, K in MIX:
        S = st.SpectralTransform(st.Spectrum(T, T), st.OctahedralGaussianGrid(nh), nlayers=K, precision="fp32")
        So = O.SpectralTransform(O.Spectrum(T, T), O.Grid(O.OCTAHEDRAL_GAUSSIAN, nh))
        c = O.random_coeffs(So.spectrum, K, seed=T)
        lt = to_lta(st, S, c)
        f_ref = st.transform(lt, S)
        a_ref = st.transform(f_ref, S)
        torch.cuda.synchronize()
        cases.append(dict(S=S, So=So, c=c, lt=lt, f_ref=np_of(f_ref), a_ref=np_of(a_ref), K=K))
    return cases


def make_batch(st, cases):
    entries, outs = [], []
    for cs in cases:
        f = st.Field.zeros(cs["S"].grid, cs["K"], device=cs["lt"].data.device)
        a = st.LowerTriangularArray.zeros(cs["S"].spectrum, cs["K"], device=cs["lt"].data.device)
        entries += [(f, cs["lt"], cs["S"]), (a, f, cs["S"])]
        outs.append((f, a))
    return st.Batch(entries), outs


def check_outputs(cases, outs, oracle=False):
    for cs, (f, a) in zip(cases, outs):
        np.testing.assert_array_equal(np_of(f), cs["f_ref"])
        np.testing.assert_array_equal(np_of(a), cs["a_ref"])
        if oracle:
            ref = cs["So"].synthesize(cs["c"])
            assert O.rel_err(np_of(f), ref) < 1e-5
            assert O.rel_err(np_of(a), cs["So"].analyze(np_of(f).astype(np.float64))) < 1e-5


def test_grouped_batch_matches_per_call(st, mixed):
    import torch
    b, outs = make_batch(st, mixed)
    b.run()
    torch.cuda.synchronize()
    check_outputs(mixed, outs, oracle=True)


def test_batch_run_each_and_graph(st, mixed):
    import torch
    b, outs = make_batch(st, mixed)
    b.run_each()
    torch.cuda.synchronize()
    check_outputs(mixed, outs)
    for f, a in outs:
        f.data.fill_(float("nan"))
        a.data.fill_(float("nan"))
    b.capture()
    b.launch()
    b.launch()
    torch.cuda.synchronize()
    check_outputs(mixed, outs)


def test_batch_autotune_keeps_results(st, mixed):
    import torch
    b, outs = make_batch(st, mixed)
    bn = b.autotune()
    assert bn in (32, 64, 128)
    for f, a in outs:
        f.data.fill_(float("nan"))
        a.data.fill_(float("nan"))
    b.run()
    torch.cuda.synchronize()
    check_outputs(mixed, outs)


def test_batch_items_sharing_a_plan(st, mixed):
    """Two syntheses on one plan in one batch: each item has its own scratch."""
    import torch
    cs = mixed[1]
    S = cs["S"]
    c2 = O.random_coeffs(cs["So"].spectrum, cs["K"], seed=99)
    lt2 = to_lta(st, S, c2)
    f1 = st.Field.zeros(S.grid, cs["K"], device=cs["lt"].data.device)
    f2 = st.Field.zeros(S.grid, cs["K"], device=cs["lt"].data.device)
    b = st.Batch([(f1, cs["lt"], S), (f2, lt2, S)])
    b.run()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(np_of(f1), cs["f_ref"])
    np.testing.assert_array_equal(np_of(f2), np_of(st.transform(lt2, S)))


def test_batch_flags(st, mixed):
    import torch
    cs = mixed[1]
    S = cs["S"]
    f = st.Field.zeros(S.grid, cs["K"], device=cs["lt"].data.device)
    f.data.fill_(1.0)
    b = st.Batch([(f, cs["lt"], S, {"unscale_coslat": True, "add": True})])
    b.run()
    torch.cuda.synchronize()
    g = st.Field.zeros(S.grid, cs["K"], device=cs["lt"].data.device)
    g.data.fill_(1.0)
    st.transform_(g, cs["lt"], S, unscale_coslat=True, add=True)
    np.testing.assert_array_equal(np_of(f), np_of(g))


def test_batch_errors(st, mixed):
    cs = mixed[1]
    big = st.LowerTriangularArray.zeros(cs["S"].spectrum, cs["K"] + 1, device=cs["lt"].data.device)
    fb = st.Field.zeros(cs["S"].grid, cs["K"] + 1, device=cs["lt"].data.device)
    with pytest.raises(st.DimensionMismatch):
        st.Batch([(fb, big, cs["S"])])


def test_plan_autotune_keeps_results(st, mixed):
    import torch
    cs = mixed[2]
    S = cs["S"]
    syn, ana = S.autotune()
    assert syn in (32, 64, 128) and ana in (32, 64, 128)
    f = st.transform(cs["lt"], S)
    a = st.transform(f, S)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(np_of(f), cs["f_ref"])
    np.testing.assert_array_equal(np_of(a), cs["a_ref"])
    St = st.SpectralTransform(st.Spectrum(32, 32), st.OctahedralGaussianGrid(24), nlayers=2, precision="bf16x3")
    assert St.autotune() in ((64, 64), (128, 128))


def test_batch_with_tensor_core_plans(st, mixed):
    """FP32 items in the grouped launches and split-FP16 / split-BF16 items as their own
    calls in one batch: run and graph replay give the bits of one transform_ per item;
    the split items stay within their tolerance of the oracle."""
    import torch
    dev = mixed[0]["lt"].data.device
    entries, refs = [], []
    for cs in mixed[:2]:                                  # FP32 T31 x 1 and T63 x 8
        f = st.Field.zeros(cs["S"].grid, cs["K"], device=dev)
        a = st.LowerTriangularArray.zeros(cs["S"].spectrum, cs["K"], device=dev)
        entries += [(f, cs["lt"], cs["S"]), (a, f, cs["S"])]
        refs += [cs["f_ref"], cs["a_ref"]]
    tc = []
    for prec, T, nh, K in [("fp16x3", 64, 48, 8), ("bf16x3", 128, 96, 16)]:
        S = st.SpectralTransform(st.Spectrum(T, T), st.OctahedralGaussianGrid(nh), nlayers=K, precision=prec)
        So = O.SpectralTransform(O.Spectrum(T, T), O.Grid(O.OCTAHEDRAL_GAUSSIAN, nh))
        c = O.random_coeffs(So.spectrum, K, seed=T + 1)
        lt = to_lta(st, S, c)
        f_ref = st.transform(lt, S)
        a_ref = st.transform(f_ref, S)
        torch.cuda.synchronize()
        f = st.Field.zeros(S.grid, K, device=dev)
        a = st.LowerTriangularArray.zeros(S.spectrum, K, device=dev)
        entries += [(f, lt, S), (a, f, S)]
        refs += [np_of(f_ref), np_of(a_ref)]
        tc.append((So, c, f, prec))
    b = st.Batch(entries)
    for how in (b.run, b.run_each):
        for out, _, _ in entries:
            out.data.zero_()
        how()
        torch.cuda.synchronize()
        for (out, _, _), ref in zip(entries, refs):
            np.testing.assert_array_equal(np_of(out), ref)
    b.capture()
    for out, _, _ in entries:
        out.data.zero_()
    b.launch()
    torch.cuda.synchronize()
    for (out, _, _), ref in zip(entries, refs):
        np.testing.assert_array_equal(np_of(out), ref)
    for So, c, f, prec in tc:
        assert O.rel_err(np_of(f), So.synthesize(c)) < (1e-6 if prec == "fp16x3" else 1e-5)


@pytest.mark.parametrize("prec", ["fp16x3", "bf16x3"])
def test_tensor_core_tile_widths_give_the_same_bits(st, prec):
    """64-column and 128-column tcgen05 tiles (48 layers: 96 columns, so 2 tiles of 64 or one
    of 128) compute every output column alike."""
    import torch
    S = st.SpectralTransform(st.Spectrum(64, 64), st.OctahedralGaussianGrid(48), nlayers=48, precision=prec)
    So = O.SpectralTransform(O.Spectrum(64, 64), O.Grid(O.OCTAHEDRAL_GAUSSIAN, 48))
    lt = to_lta(st, S, O.random_coeffs(So.spectrum, 48, seed=9))
    out = {}
    for cols in (128, 64):
        S.set_tile_columns(cols)
        f = st.transform(lt, S)
        a = st.transform(f, S)
        torch.cuda.synchronize()
        out[cols] = (f.data.clone(), a.data.clone())
    assert S.device_status() == 0
    assert torch.equal(out[64][0], out[128][0]) and torch.equal(out[64][1], out[128][1])
    from speedytransforms._lib import ShtError
    with pytest.raises(ShtError):
        S.set_tile_columns(32)
