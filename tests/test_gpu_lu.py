"""Device FP64 blocked complex LU vs numpy and the oracle's LU (dense.rs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 127, 200, 513])
def test_lu_matches_numpy(fh, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    x = fh.lu_solve(a, b)
    want = np.linalg.solve(a, b)
    assert np.max(np.abs(x - want)) / np.max(np.abs(want)) < 1e-10
    res = np.max(np.abs(a @ x - b)) / (np.max(np.abs(a)) * np.max(np.abs(x)))
    assert res < 1e-14 * max(1, n / 8)


def test_lu_matches_oracle_pivoting(fh, oracle):
    rng = np.random.default_rng(5)
    n = 300
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a[:, 7] *= 1e-8  # forces interchanges
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x = fh.lu_solve(a, b)
    xo = oracle.lu_solve(a, b)
    assert np.max(np.abs(x - xo)) / np.max(np.abs(xo)) < 1e-10


def test_lu_vector_rhs_shape(fh):
    a = np.array([[2.0, 1.0], [1.0, 3.0]], dtype=complex)
    x = fh.lu_solve(a, np.array([1.0, 2.0]))
    assert x.shape == (2,)
    assert np.allclose(a @ x, [1.0, 2.0])


def test_singular_is_reported(fh):
    a = np.zeros((5, 5), dtype=complex)
    with pytest.raises(fh.Singular):
        fh.lu_solve(a, np.ones(5))
    a = np.eye(70, dtype=complex)
    a[69, 69] = 0.0
    with pytest.raises(fh.Singular):
        fh.lu_solve(a, np.ones(70))


def test_shape_errors(fh):
    with pytest.raises(fh.InvalidArgument):
        fh.lu_solve(np.ones((2, 3)), np.ones(2))
    with pytest.raises(fh.InvalidArgument):
        fh.lu_solve(np.eye(3), np.ones(2))
