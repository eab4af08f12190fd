"""The engine's dense solver (the partial-pivot LU solves of the Dyson step and the
bootstrap, src/dyson_step.h:65, :163, :252, src/dyson_boot.h:61, :170) against numpy,
through the C ABI, at the shapes the engine solves and at ragged ones:

* one 320 x 320 system with 64 right-hand sides (the retarded / lesser start block at
  nao = 64, k = 5) and one with 320 (the bootstrap inverse), spread over a cluster of CTAs;
* a batch of 64 x 64 inverses (the cached time-local Dyson matrices);
* sizes whose augmented width does not divide evenly over the cluster, a single row, and
  a system larger than the shared memory of one cluster (the global-memory path);
* a singular system (NEDY_ERR_SINGULAR).

Tolerance: max |X - X_numpy| <= 1e-11 * cond-scaled max |X_numpy| (the systems are
diagonally shifted to condition numbers of order 10).
"""
import ctypes as C

import numpy as np
import pytest

from nedyson_b200 import _lib, api

pytestmark = pytest.mark.gpu


def _systems(n, nrhs, nb, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((nb, n, n)) + 1j * rng.standard_normal((nb, n, n))
    A += (2.0 * np.sqrt(n)) * np.exp(1j * rng.uniform(0, 2 * np.pi, (nb, 1, 1))) * np.eye(n)
    # a row permutation so that partial pivoting has work to do
    A = A[:, rng.permutation(n), :]
    B = rng.standard_normal((nb, n, nrhs)) + 1j * rng.standard_normal((nb, n, nrhs))
    return np.ascontiguousarray(A), np.ascontiguousarray(B)


def _solve(ctx, A, B):
    nb, n, nrhs = B.shape
    A0 = A.copy()
    X = B.copy()
    st = _lib.lib().nedy_dense_solve(ctx.h, n, nrhs, nb, A.ctypes.data_as(C.c_void_p), X.ctypes.data_as(C.c_void_p))
    assert np.array_equal(A, A0)  # A is left as it was
    return st, X


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(8, 8, 4, 5, 1.0, 0.01)
    yield c
    c.close()


@pytest.mark.parametrize("n,nrhs,nb", [(320, 64, 1), (320, 320, 1), (64, 64, 7), (160, 32, 1), (130, 3, 1),
                                       (201, 1, 2), (1, 5, 3), (20, 4, 5), (700, 9, 1)])
def test_dense_solve_matches_numpy(ctx, n, nrhs, nb):
    A, B = _systems(n, nrhs, nb, seed=n * 31 + nrhs + nb)
    st, X = _solve(ctx, A, B)
    assert st == _lib.NEDY_OK, _lib.lib().nedy_last_error()
    ref = np.linalg.solve(A, B)
    err = np.abs(X - ref).max() / np.abs(ref).max()
    print(f"dense solve n={n} nrhs={nrhs} nb={nb}: {err:.2e}")
    assert err < 1e-11


def test_dense_solve_singular(ctx):
    A, B = _systems(64, 8, 1, seed=5)
    A[0, :, 3] = 0.0  # a zero column
    st, _ = _solve(ctx, A, B)
    assert st == 7  # NEDY_ERR_SINGULAR
    # the context stays usable
    A, B = _systems(64, 8, 1, seed=6)
    st, X = _solve(ctx, A, B)
    assert st == _lib.NEDY_OK
    assert np.abs(X - np.linalg.solve(A, B)).max() < 1e-10
