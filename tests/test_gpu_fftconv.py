"""The pFFT grid convolution without a library FFT (fh_fftconv.cu: pruned
mixed-radix Stockham transforms in shared memory) against numpy's FFT of the
same aperiodic convolution (the kernel 1 / (h |d|), zero at d = 0, on the
padded torus m_a >= 2 n_a - 1, fft.rs:1-30 of the reference): FP64 to 1e-12
and FP32 to 2e-6 (max-norm relative), over axis lengths with every radix
(2, 3, 4, 5), single-point axes, an odd number of fields, and a long axis."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def smooth(n):
    m = max(n, 1)
    while True:
        r = m
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def reference(q, m, h):
    n = q.shape[1:]
    idx = [np.arange(mm) for mm in m]
    d = [np.where(i < nn, i, np.where(i + nn > mm, i - mm, 10 ** 9)) for i, nn, mm in zip(idx, n, m)]
    D0, D1, D2 = np.meshgrid(*d, indexing="ij")
    valid = (np.abs(D0) < 10 ** 8) & (np.abs(D1) < 10 ** 8) & (np.abs(D2) < 10 ** 8)
    r = np.sqrt((D0.astype(float) ** 2 + D1.astype(float) ** 2 + D2.astype(float) ** 2))
    K = np.where(valid & (r > 0), 1.0 / (h * np.where(r > 0, r, 1.0)), 0.0)
    spec = np.fft.fftn(K)
    out = []
    for f in range(q.shape[0]):
        g = np.zeros(m)
        g[:n[0], :n[1], :n[2]] = q[f]
        out.append(np.real(np.fft.ifftn(np.fft.fftn(g) * spec))[:n[0], :n[1], :n[2]])
    return np.array(out)


@pytest.mark.parametrize("n,fields", [((3, 4, 5), 2), ((7, 1, 13), 3), ((1, 1, 1), 1), ((20, 30, 2), 4),
                                      ((60, 70, 8), 2), ((2, 600, 3), 1), ((33, 17, 9), 2)])
@pytest.mark.parametrize("fp32", [False, True])
def test_grid_convolution_matches_numpy(fh, n, fields, fp32):
    m = [smooth(2 * a - 1) for a in n]
    rng = np.random.default_rng(sum(n) + fields)
    q = rng.standard_normal((fields,) + tuple(n))
    h = 2.5e-5
    got = fh.grid_convolution(q, m, h, fp32=fp32)
    want = reference(q, m, h)
    if n == (1, 1, 1):  # a single point has no partner: the potential is zero
        assert np.all(got == 0.0)
        return
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert err < (2e-6 if fp32 else 1e-12), err


def test_larger_padding_than_needed_gives_the_same_result(fh):
    n = (9, 10, 4)
    rng = np.random.default_rng(5)
    q = rng.standard_normal((2,) + n)
    a = fh.grid_convolution(q, [smooth(2 * x - 1) for x in n], 1e-5)
    b = fh.grid_convolution(q, [32, 45, 16], 1e-5)
    assert np.max(np.abs(a - b)) / np.max(np.abs(a)) < 1e-12
