"""fh_lu_solve_c64_noalloc: the FP64 LU solve for callers that cannot
allocate device memory while they solve (an application whose device memory
all belongs to its own pool, or a loop that must not cudaMalloc/cudaFree).

The caller owns the device buffers (here: torch tensors); the entry point
itself allocates nothing and keeps its scratch in a fixed device array.  Its
result must equal the allocating entry point's (fh_lu_solve_c64) and
numpy.linalg.solve within the LU tests' tolerance, on two calls in a row (the
second call sees the array the first one left behind), and the device's free
memory must not move across its calls.  This file is collected last on
purpose.
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


def _system(n, nrhs, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    return a, b


def _rel(got, want):
    return np.max(np.abs(got - want)) / np.max(np.abs(want))


def test_noalloc_lu_matches_allocating_lu_and_numpy_twice(fh):
    import torch
    N, fn = _lib()
    for call, (n, nrhs) in enumerate([(300, 2), (129, 1)]):
        a, b = _system(n, nrhs, 100 + call)
        want = np.linalg.solve(a, b)
        alloc = fh.lu_solve(a, b)  # the allocating entry point
        da = _device_complex(torch, a)
        db = _device_complex(torch, b)
        torch.cuda.synchronize()
        info = N.ErrorInfo()
        st = fn(da.data_ptr(), n, db.data_ptr(), nrhs, None, ctypes.byref(info))
        assert st == N.OK, N.last_error()
        torch.cuda.synchronize()
        got = _from_device(db, n, nrhs)
        assert _rel(got, want) < RTOL
        assert _rel(got, alloc) < RTOL


def test_noalloc_lu_leaves_device_memory_untouched(fh):
    """No cudaMalloc (the driver's free memory stays put) and nothing taken from
    the library's own pool (its idle memory is released first, so a pool
    allocation would have to map new memory)."""
    import torch
    N, fn = _lib()
    n, nrhs = 2000, 3
    a, b = _system(n, nrhs, 7)
    want = np.linalg.solve(a, b)
    # Set-up call: loads the kernels and looks up the scratch array's address.
    da, db = _device_complex(torch, a), _device_complex(torch, b)
    info = N.ErrorInfo()
    assert fn(da.data_ptr(), n, db.data_ptr(), nrhs, None, ctypes.byref(info)) == N.OK, N.last_error()
    inputs = [(_device_complex(torch, a), _device_complex(torch, b)) for _ in range(2)]
    torch.cuda.synchronize()
    fh.release_cached_memory()
    free_before = torch.cuda.mem_get_info()[0]
    for da, db in inputs:
        assert fn(da.data_ptr(), n, db.data_ptr(), nrhs, None, ctypes.byref(info)) == N.OK, N.last_error()
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    for _, db in inputs:
        assert _rel(_from_device(db, n, nrhs), want) < RTOL


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
