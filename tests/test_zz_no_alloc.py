"""nedy_hf_decomp_noalloc against nedy_hf_decomp, through the C ABI.

The no-allocation entry point keeps its intermediates in one static device
array shared by every call, so two calls in a row (different time slices,
different densities) must both reproduce the allocating entry point.
"""
import numpy as np
import pytest

from nedyson_b200 import _lib, api

pytestmark = pytest.mark.gpu

TOL = 1e-10
NEDY_ERR_ARG = 1


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


def _hermitian(rng, n):
    x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return 0.5 * (x + x.conj().T)


@pytest.mark.parametrize("nao,naux", [(6, 11), (64, 256)])
def test_hf_noalloc_matches_hf_decomp_twice(nao, naux):
    rng = np.random.default_rng(1000 + nao)
    nt = 4
    ctx = api.Context(nt, 4, nao, 1, 1.0, 0.01)
    V = rng.standard_normal((nao, nao, naux)) * 0.1
    V = 0.5 * (V + V.transpose(1, 0, 2))
    api.molGF2SolverDecomp(ctx, V)
    h0 = np.stack([_hermitian(rng, nao) for _ in range(nt + 1)])
    h_ref = api.hmf_buffer(ctx, nao, h0)
    h_new = api.hmf_buffer(ctx, nao, h0)
    lib = _lib.lib()
    for tstp in (3, 1):
        rho = api.DeviceBuffer.from_array(ctx, np.ascontiguousarray(_hermitian(rng, nao)))
        _lib.check(lib.nedy_hf_decomp(ctx.h, tstp, h_ref.h, rho.h))
        _lib.check(lib.nedy_hf_decomp_noalloc(ctx.h, tstp, h_new.h, rho.h))
        a = h_new.download((nt + 1, nao, nao))
        b = h_ref.download((nt + 1, nao, nao))
        assert rel(a[tstp], b[tstp]) < TOL
        assert np.max(np.abs(b[tstp] - h0[tstp])) > 0.0  # the update did something
        assert np.array_equal(np.delete(a, [1, 3], axis=0), np.delete(h0, [1, 3], axis=0))
    ctx.close()


def test_hf_noalloc_rejects_sizes_beyond_scratch():
    nao, naux = 64, 512  # 16 * 64 * 64 * 512 bytes alone exceed the 24 MiB array
    ctx = api.Context(2, 4, nao, 1, 1.0, 0.01)
    api.molGF2SolverDecomp(ctx, np.zeros((nao, nao, naux)))
    h = api.hmf_buffer(ctx, nao, np.zeros((3, nao, nao), np.complex128))
    rho = api.DeviceBuffer.from_array(ctx, np.zeros((nao, nao), np.complex128))
    st = _lib.lib().nedy_hf_decomp_noalloc(ctx.h, 0, h.h, rho.h)
    assert st == NEDY_ERR_ARG
    assert b"scratch" in _lib.lib().nedy_last_error()
    ctx.close()
