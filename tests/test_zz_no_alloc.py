"""fh_lu_solve_c64_noalloc: the FP64 LU solve for callers that cannot
allocate device memory while they solve (an application whose device memory
all belongs to its own pool, or a loop that must not cudaMalloc/cudaFree).

The caller owns the device buffers (here: torch tensors); the entry point
itself allocates nothing and keeps its scratch in a fixed device array.  Its
result must equal the allocating entry point's (fh_lu_solve_c64) within the
LU tests' tolerance, on two calls in a row (the second call sees the array
the first one left behind).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10  # as tests/test_gpu_lu.py


def _lib():
    from fasterhenry_b200 import _native as N
    lib = N.load()
    fn = lib.fh_lu_solve_c64_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                   ctypes.POINTER(N.ErrorInfo)]
    fn.restype = ctypes.c_int
    return N, fn


def _device_complex(torch, z):
    """Column-major complex128 matrix as an interleaved float64 CUDA tensor."""
    zf = np.asfortranarray(z.reshape(z.shape[0], -1))
    flat = np.ascontiguousarray(zf.T).reshape(-1)  # column-major order
    inter = np.stack([flat.real, flat.imag], axis=1).reshape(-1)
    return torch.tensor(inter, dtype=torch.float64, device="cuda")


def _from_device(t, rows, cols):
    v = t.cpu().numpy().reshape(-1, 2)
    flat = v[:, 0] + 1j * v[:, 1]
    return flat.reshape(cols, rows).T


def test_noalloc_lu_matches_allocating_lu_twice(fh):
    import torch
    N, fn = _lib()
    for call, (n, nrhs) in enumerate([(300, 2), (129, 1)]):
        rng = np.random.default_rng(100 + call)
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
        want = fh.lu_solve(a, b)  # the allocating entry point
        da = _device_complex(torch, a)
        db = _device_complex(torch, b)
        torch.cuda.synchronize()
        info = N.ErrorInfo()
        st = fn(da.data_ptr(), n, db.data_ptr(), nrhs, None, ctypes.byref(info))
        assert st == N.OK, N.last_error()
        torch.cuda.synchronize()
        got = _from_device(db, n, nrhs)
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < RTOL


def test_noalloc_rejects_orders_beyond_the_limit():
    N, fn = _lib()
    info = N.ErrorInfo()
    st = fn(None, 65537, None, 1, None, ctypes.byref(info))
    assert st == N.ERR_INVALID_ARGUMENT
    assert "exceeds the maximum of 65536" in N.last_error()


def test_noalloc_reports_a_singular_matrix(fh):
    import torch
    N, fn = _lib()
    n = 70
    a = np.eye(n, dtype=complex)
    a[n - 1, n - 1] = 0.0
    da = _device_complex(torch, a)
    db = _device_complex(torch, np.ones((n, 1), dtype=complex))
    info = N.ErrorInfo()
    assert fn(da.data_ptr(), n, db.data_ptr(), 1, None, ctypes.byref(info)) == N.ERR_SINGULAR
