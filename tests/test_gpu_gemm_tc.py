"""The LU trailing update A22 -= L21 U12 (complex FP32 storage) on the tensor
cores (split-BF16 x3) and in FP32 SIMT, against an FP64 numpy product of the
same FP32 inputs.

Tolerance: |C - C_ref| <= tol * (|L21| |U12| + |C|) entry-wise, with
tol = 2e-5 for the split-BF16 x3 form (three BF16 products per real product,
about 2^-17 relative each, FP32 accumulation) and 2e-6 for FP32 SIMT.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(fh, a, k0, nb, mode):
    from fasterhenry_b200 import _native as N
    from fasterhenry_b200.api import _check
    count, m = a.shape[0], a.shape[1]
    buf = np.ascontiguousarray(np.transpose(a, (0, 2, 1)).astype(np.complex64))  # column-major per matrix
    info = N.ErrorInfo()
    _check(N.load().fh_test_trailing_update(buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), m, count, k0, nb,
                                            mode, ctypes.byref(info)), info)
    return np.transpose(buf, (0, 2, 1))


def reference(a, k0, nb):
    a64 = a.astype(np.complex128)
    out = a64.copy()
    b = k0 + nb
    for f in range(a.shape[0]):
        out[f, b:, b:] -= a64[f, b:, k0:b] @ a64[f, k0:b, b:]
    bound = np.zeros(a.shape)
    for f in range(a.shape[0]):
        bound[f, b:, b:] = np.abs(a64[f, b:, k0:b]) @ np.abs(a64[f, k0:b, b:]) + np.abs(a64[f, b:, b:])
    return out, bound


@pytest.mark.parametrize("m,count,k0,nb", [(200, 1, 0, 64), (300, 2, 64, 64), (457, 3, 128, 64), (1000, 1, 0, 32),
                                           (130, 2, 0, 16)])
@pytest.mark.parametrize("mode,tol", [(1, 2e-5), (0, 2e-6)])
def test_trailing_update(fh, m, count, k0, nb, mode, tol):
    rng = np.random.default_rng(m + count + k0)
    a = (rng.standard_normal((count, m, m)) + 1j * rng.standard_normal((count, m, m))).astype(np.complex64)
    a[:, :, k0:k0 + nb] *= 0.3  # multipliers below one, as partial pivoting makes them
    ref, bound = reference(a, k0, nb)
    got = run(fh, a, k0, nb, mode)
    b = k0 + nb
    # columns/rows outside the trailing block are untouched
    assert np.array_equal(got[:, :b, :], a[:, :b, :])
    assert np.array_equal(got[:, :, :b], a[:, :, :b])
    err = np.abs(got[:, b:, b:] - ref[:, b:, b:]) / bound[:, b:, b:]
    assert err.max() < tol, err.max()


@pytest.mark.parametrize("m,count,k0,nb", [(1200, 1, 64, 512), (900, 3, 0, 256), (300, 2, 16, 128), (130, 2, 0, 16),
                                           (777, 2, 100, 512), (1500, 1, 0, 1024)])
def test_packed_update(fh, m, count, k0, nb):
    """Persistent tensor-core kernel from packed split-BF16 operands (mode 2),
    including deep K (512, 1024), ragged tiles and a batch."""
    rng = np.random.default_rng(7 * m + count + k0)
    a = (rng.standard_normal((count, m, m)) + 1j * rng.standard_normal((count, m, m))).astype(np.complex64)
    a[:, :, k0:k0 + nb] *= 0.3
    ref, bound = reference(a, k0, nb)
    got = run(fh, a, k0, nb, 2)
    b = k0 + nb
    assert np.array_equal(got[:, :b, :], a[:, :b, :])
    assert np.array_equal(got[:, :, :b], a[:, :, :b])
    err = np.abs(got[:, b:, b:] - ref[:, b:, b:]) / bound[:, b:, b:]
    assert err.max() < 2e-5, err.max()
