"""The algebra of the tensor-core prime stage (csrc/sht_prime_tc.cu), checked in numpy.

For a ring of n = p nb points the kernel computes the first Stockham stage, nb DFTs of
length p over x_q = z[i0 + q nb], as two real matrix products with the (h + 1)^2 cosine and
sine matrices (h = (p - 1) / 2) over u_q = x_q + x_(p-q) (u_0 = x_0) and v_q = x_q - x_(p-q)
(v_0 = 0), and writes y_r = A_r -+ i B_r and y_(p-r) = A_r +- i B_r (forward / inverse) to
y[i0 p + r]. The FFT kernel then runs the remaining radices from Ns = p. These tests
restate that stage, finish the transform with the remaining radix-nb stage of a Stockham
FFT, and compare with numpy's FFT; they also bound the TF32 hi/lo split of the matrices.
"""
import numpy as np
import pytest


def tf32(x):
    """Round to the 11-bit significand of TF32, to nearest with ties away from zero (the
    kernel's integer trick on the FP32 bits)."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def first_stage(z, p, inverse):
    """y[i0 p + r] of the first stage, from the kernel's u/v products (FP64)."""
    n = z.size
    nb = n // p
    h = (p - 1) // 2
    r = np.arange(h + 1)
    q = np.arange(h + 1)
    C = np.cos(2 * np.pi * ((np.outer(r, q)) % p) / p)
    S = np.sin(2 * np.pi * ((np.outer(r, q)) % p) / p)
    y = np.zeros(n, complex)
    for i0 in range(nb):
        x = z[i0 + nb * np.arange(p)]
        u = np.empty(h + 1, complex)
        v = np.empty(h + 1, complex)
        u[0], v[0] = x[0], 0
        u[1:] = x[1:h + 1] + x[p - np.arange(1, h + 1)]
        v[1:] = x[1:h + 1] - x[p - np.arange(1, h + 1)]
        A = C @ u
        B = S @ v
        yr = A - 1j * B if not inverse else A + 1j * B
        ypr = A + 1j * B if not inverse else A - 1j * B
        y[i0 * p + r] = yr
        y[i0 * p + p - r[1:]] = ypr[1:]
    return y


def finish(y, p, inverse):
    """The remaining Stockham stage of radix nb at Ns = p: out[k + p s] = sum_i0
    w_n^(+-i0 k) w_nb^(+-i0 s) y[i0 p + k]."""
    n = y.size
    nb = n // p
    sgn = 1 if inverse else -1
    out = np.zeros(n, complex)
    for k in range(p):
        col = y[np.arange(nb) * p + k] * np.exp(sgn * 2j * np.pi * np.arange(nb) * k / n)
        out[k + p * np.arange(nb)] = np.exp(sgn * 2j * np.pi * np.outer(np.arange(nb), np.arange(nb)) / nb).T @ col
    return out


@pytest.mark.parametrize("p,nb", [(67, 4), (97, 8), (131, 4), (383, 4)])
@pytest.mark.parametrize("inverse", [False, True])
def test_first_stage_then_radix_nb_is_the_dft(p, nb, inverse):
    rng = np.random.default_rng(p + nb)
    z = rng.standard_normal(p * nb) + 1j * rng.standard_normal(p * nb)
    got = finish(first_stage(z, p, inverse), p, inverse)
    ref = np.fft.ifft(z) * z.size if inverse else np.fft.fft(z)
    assert np.max(np.abs(got - ref)) < 1e-9 * np.max(np.abs(ref))


@pytest.mark.parametrize("p", [67, 193, 383])
def test_tf32_split_keeps_22_bits(p):
    h = (p - 1) // 2
    rq = np.outer(np.arange(h + 1), np.arange(h + 1)) % p
    for f in (np.cos, np.sin):
        m = f(2 * np.pi * rq / p)
        hi = tf32(m)
        lo = tf32(m - hi.astype(np.float64))
        err = np.abs(hi.astype(np.float64) + lo.astype(np.float64) - m)
        # two 11-bit pieces: the remainder is below 2^-22 of each entry (plus FP32 rounding)
        assert np.all(err <= 2.0 ** -22 * np.abs(m) + 2.0 ** -40)
