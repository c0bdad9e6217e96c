"""Several spectral operators in one launch (sht_operators) against the single calls.

Each operator of a set gives the bits of its single call (curl, divergence, Laplacian,
inverse Laplacian, gradient, UV_from_vordiv, with flipsign/add/radius), including chains
of operators accumulating into the same output in list order; sets that alias an input
with an output, or outputs with each other, are rejected before any launch.
"""
import pytest

pytestmark = pytest.mark.gpu

R = 6.371e6


@pytest.fixture(scope="module")
def st():
    import speedytransforms as st
    return st


def _setup(st, T, K, nh=None):
    import torch
    sp = st.Spectrum(T + 1, T)
    S = st.SpectralTransform(sp, st.OctahedralGaussianGrid(nh or st.get_nlat_half(T)), nlayers=K)
    g = torch.Generator(device="cuda").manual_seed(T)

    def field():
        return st.LowerTriangularArray(torch.randn((K, sp.nlm), dtype=torch.complex64, device="cuda", generator=g), sp)
    return S, field


@pytest.mark.parametrize("T,K", [(31, 4), (255, 22)])
def test_each_operator_equals_its_single_call(st, T, K):
    import torch
    S, field = _setup(st, T, K)
    u, v, p = field(), field(), field()
    outs_single = [field() for _ in range(8)]
    outs_batch = [st.LowerTriangularArray(o.data.clone(), S.spectrum) for o in outs_single]
    st.curl_(outs_single[0], u, v, S, add=True, radius=R)
    st.divergence_(outs_single[1], u, v, S, flipsign=True, radius=R)
    st.laplace_(outs_single[2], p, S, add=True, flipsign=True)
    st.laplace_(outs_single[3], p, S, inverse=True, radius=R)
    st.gradient_(outs_single[4], outs_single[5], p, S, radius=R)
    st.UV_from_vordiv_(outs_single[6], outs_single[7], u, v, S, radius=R)
    ops = (st.Operators(S)
           .curl(outs_batch[0], u, v, add=True, radius=R)
           .divergence(outs_batch[1], u, v, flipsign=True, radius=R)
           .laplace(outs_batch[2], p, add=True, flipsign=True)
           .laplace(outs_batch[3], p, inverse=True, radius=R)
           .gradient(outs_batch[4], outs_batch[5], p, radius=R)
           .UV_from_vordiv(outs_batch[6], outs_batch[7], u, v, radius=R))
    ops()
    torch.cuda.synchronize()
    for x, y in zip(outs_single, outs_batch):
        assert torch.equal(x.data, y.data)


def test_accumulation_chain_in_order(st):
    """curl, divergence (flipsign) and a Laplacian all adding into one output, then an
    operator with a different layer count: the separate calls' result, bit for bit."""
    import torch
    S, field = _setup(st, 63, 8)
    u, v, p = field(), field(), field()
    ref = field()
    out = st.LowerTriangularArray(ref.data.clone(), S.spectrum)
    st.curl_(ref, u, v, S, add=True)
    st.divergence_(ref, u, v, S, add=True, flipsign=True)
    st.laplace_(ref, p, S, add=True)
    part = st.LowerTriangularArray(field().data[:3], S.spectrum)
    part_ref = st.LowerTriangularArray(part.data.clone(), S.spectrum)
    st.laplace_(part_ref, st.LowerTriangularArray(p.data[:3], S.spectrum), S, inverse=True)
    (st.Operators(S).curl(out, u, v, add=True).divergence(out, u, v, add=True, flipsign=True)
     .laplace(out, p, add=True).laplace(part, st.LowerTriangularArray(p.data[:3], S.spectrum), inverse=True))()
    torch.cuda.synchronize()
    assert torch.equal(out.data, ref.data)
    assert torch.equal(part.data, part_ref.data)


def test_aliasing_rejected(st):
    import torch
    from speedytransforms import _lib
    S, field = _setup(st, 31, 4)
    nlm = S.spectrum.nlm
    u, v, o = field(), field(), field()
    before = o.data.clone()
    with pytest.raises(_lib.ShtError):     # an input that is an output of the set
        st.Operators(S).curl(o, u, v).laplace(u, v)()
    flat = o.data.reshape(-1)
    a = st.LowerTriangularArray(flat[: 3 * nlm].reshape(3, nlm), S.spectrum)
    b = st.LowerTriangularArray(flat[1: 1 + 3 * nlm].reshape(3, nlm), S.spectrum)
    u3 = st.LowerTriangularArray(u.data[:3], S.spectrum)
    with pytest.raises(_lib.ShtError):     # overlapping outputs that are not the same array
        st.Operators(S).laplace(a, u3).laplace(b, u3)()
    torch.cuda.synchronize()
    assert torch.equal(o.data, before)     # nothing ran
