"""Sigma's two-time history in pinned host memory (nedy_gf_create_host_history): the kernels
read and write the lesser and retarded triangles in place over the host link, so a
trajectory stepped with a host-resident Sigma equals the same trajectory with Sigma in
device memory to the last bit of the arithmetic (the same values at other addresses).
Restricted density-fitted GF2, nao=5, with a windowed G as in a long run, with the residual
exit and with the fixed corrector loop."""
import ctypes as C

import numpy as np
import pytest

from nedyson_b200 import _lib
from nedyson_b200.inputs import make_problem
from nedyson_b200.simulation import DecompSimulation


def test_host_history_argument_checks():
    """Without a device: the sizes are checked before any allocation."""
    L = _lib.lib()
    out = C.c_void_p()
    assert L.nedy_gf_create_host_history(None, 20, 4, 2, -1, C.byref(out)) == 1
    flag = C.c_int(7)
    assert L.nedy_gf_host_history(None, C.byref(flag)) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("fixed", [False, True])
def test_host_sigma_trajectory_matches_device(fixed):
    p = make_problem(5, 15, seed=37)
    kw = dict(nt=36, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=3, drive_kind="gauss",
              drive_kw=dict(E0=0.1, t0=0.3, sigma=0.1))
    dev = DecompSimulation(p, **kw)
    host = DecompSimulation(p, g_window=12, sigma_host=True, **kw)
    assert not dev.Sigma.host_history and host.Sigma.host_history and host.G.window == 12
    for s in (dev, host):
        s.free_gf()
        s.do_boot(max_iter=10, tol=0.0)
    worst = 0.0
    for t in range(6, 37):
        for s in (dev, host):
            if fixed:
                s.do_tstp(t)
            else:
                s.do_tstp_tol(t, 1e-10, 5)
        for a, b in ((dev.G.ret_row(t), host.G.ret_row(t)), (dev.G.les_col(t), host.G.les_col(t)),
                     (dev.G.tv_row(t), host.G.tv_row(t))):
            worst = max(worst, float(np.abs(a - b).max()))
    # Sigma's history itself, read back from host memory through the same entry point
    ntri = 37 * 38 // 2
    for comp in (_lib.RET, _lib.LES):
        worst = max(worst, float(np.abs(dev.Sigma.download(comp, 0, ntri) - host.Sigma.download(comp, 0, ntri)).max()))
    print(f"host-resident vs device Sigma over 31 steps: max |difference| {worst:.3e}")
    assert worst <= 1e-13
    for s in (dev, host):
        s.ctx.close()
