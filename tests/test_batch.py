"""Batched stepping of independent simulations of uneven size (nedy_batch_tstp) against the
oracle: every instance of the batch must follow its own reference trajectory
(DecompSimulation::do_tstp, reference src/molNEsim_decomp_impl.h:85-104) to 1e-10, as if
it had been stepped alone."""
import numpy as np
import pytest

from nedyson_b200.simulation import BatchSimulation, batch_problems
from simref import OracleDecompSim

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))


def test_batch_matches_oracle_per_instance():
    probs = batch_problems(6, seed=5, nao_range=(2, 9), amp_range=(0.2, 0.6), freq_range=(1.0, 3.0))
    kw = dict(nt=12, ntau=16, beta=10.0, dt=0.02, k=5, corr_steps=2)
    b = BatchSimulation(probs, workers=3, workspace_bytes=64 << 20, **kw)
    b.boot(max_iter=10)
    refs = []
    for p, dkw in probs:
        r = OracleDecompSim(p, drive_kind="sin", drive_kw=dkw, **kw)
        r.free_gf()
        r.do_boot(max_iter=10)
        refs.append(r)
    for t in range(6, 13):
        its = b.do_tstp(t)
        assert its == [2] * len(probs)
        for r in refs:
            r.do_tstp(t)
    for s, r in zip(b.sims, refs):
        g = s.G.to_host()
        for comp in ("les", "ret", "tv"):
            e = rel(getattr(g, comp), getattr(r.G, comp))
            assert e < 1e-10, (s.p.nao, comp, e)
    # the residual-exit form runs through the same pool
    its = b.do_tstp(12, tol=1e-9)
    assert all(1 <= i <= 2 for i in its)
    b.close()


def test_batch_rejects_bad_step():
    from nedyson_b200 import _lib
    probs = batch_problems(2, seed=6, nao_range=(2, 3))
    b = BatchSimulation(probs, nt=8, ntau=8, beta=5.0, dt=0.02, k=5, corr_steps=1, workspace_bytes=32 << 20)
    rc = _lib.lib().nedy_batch_tstp(b.h, 3, 1, 0.0, None)  # tstp <= k
    assert rc == 1 and b"tstp" in _lib.lib().nedy_last_error()
    b.close()
