"""Checkpoint and resume through the HDF5 output (nedyson_b200/checkpoint.py).

A run saved after step t and loaded into a fresh simulation of the same sizes must
continue exactly like the uninterrupted run (up to the order of FP64 atomic sums), for
the restricted, unrestricted and full-U drivers; the file holds the reference's
save() layout (src/molNEsim_decomp_impl.h:107-122, src/greens.cpp:202-239).
"""
import numpy as np
import pytest

from nedyson_b200 import checkpoint
from nedyson_b200.h5io import H5File
from nedyson_b200.inputs import make_problem
from nedyson_b200.simulation import DecompSimulation, DecompSpinSimulation, FullSimulation

pytestmark = pytest.mark.gpu


def _rows(sim, t0, t1):
    Gs = sim.G if isinstance(sim.G, list) else [sim.G]
    out = []
    for g in Gs:
        h = g.to_host()
        out.append(np.concatenate([np.concatenate([h.les_col(t).ravel(), h.ret_row(t).ravel(), h.tv[t].ravel()])
                                   for t in range(t0, t1 + 1)]))
    return out


@pytest.mark.parametrize("kind", ["restricted", "unrestricted", "full"])
def test_save_load_resume(kind, tmp_path):
    spin = kind == "unrestricted"
    p = make_problem(4, 8, seed=23, spin=spin)
    kw = dict(nt=14, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=2, drive_kind="gauss",
              drive_kw=dict(E0=0.5, t0=0.15, sigma=0.05))
    Sim = {"restricted": DecompSimulation, "unrestricted": DecompSpinSimulation, "full": FullSimulation}[kind]
    a = Sim(p, **kw)
    a.free_gf()
    a.do_boot(max_iter=10)
    for t in range(6, 11):
        a.do_tstp(t)
    path = str(tmp_path / "run.h5")
    checkpoint.save(a, path, t_last=10)
    for t in range(11, 15):
        a.do_tstp(t)
    ref = _rows(a, 11, 14)
    f = H5File(path)
    assert f["/solve/last_tstp"] == 10 and f["/solve/params/CorrSteps"] == 2
    g = "/G/up" if spin else "/G"
    assert f[g + "/nt"] == 14 and f[g + "/GL"].shape == ((15 * 16 // 2) * 16,)
    assert f["/energy/potential"].shape == (15,)
    b = Sim(p, **kw)
    assert checkpoint.load(b, path) == 10
    for t in range(11, 15):
        b.do_tstp(t)
    for x, y in zip(_rows(b, 11, 14), ref):
        assert np.abs(x - y).max() <= 1e-12 * max(1.0, np.abs(y).max())
    a.ctx.close()
    b.ctx.close()
