"""Windowed Green's function (only the last W time steps of G^R and G^< on the device,
Sigma whole): a trajectory stepped with a windowed G equals the same trajectory with the
full triangles, row by row, to the last bit of the arithmetic (the kernels read the same
values; only their addresses differ).  Restricted density-fitted GF2, nao=5, with the
residual exit and with the fixed corrector loop."""
import numpy as np
import pytest

from nedyson_b200 import _lib, api
from nedyson_b200.inputs import make_problem
from nedyson_b200.simulation import DecompSimulation


def test_window_argument_checks():
    """Without a device: the sizes are checked before any allocation."""
    import ctypes as C
    L = _lib.lib()
    out = C.c_void_p()
    assert L.nedy_gf_create_windowed(None, 20, 4, 2, -1, 16, C.byref(out)) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("fixed", [False, True])
def test_windowed_trajectory_matches_full(fixed):
    p = make_problem(5, 15, seed=31)
    kw = dict(nt=40, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=3, drive_kind="gauss",
              drive_kw=dict(E0=0.1, t0=0.3, sigma=0.1))
    full = DecompSimulation(p, **kw)
    win = DecompSimulation(p, g_window=12, **kw)
    assert full.G.window == 0 and win.G.window == 12
    for s in (full, win):
        s.free_gf()
        s.do_boot(max_iter=10, tol=0.0)
    worst = 0.0
    for t in range(6, 41):
        for s in (full, win):
            if fixed:
                s.do_tstp(t)
            else:
                s.do_tstp_tol(t, 1e-10, 5)
        for a, b in ((full.G.ret_row(t), win.G.ret_row(t)), (full.G.les_col(t), win.G.les_col(t)),
                     (full.G.tv_row(t), win.G.tv_row(t))):
            worst = max(worst, float(np.abs(a - b).max()))
    print(f"windowed vs full G over 35 steps: max |difference| {worst:.3e}")
    assert worst <= 1e-13
    # rows older than the window are gone from the device: reading them is refused
    with pytest.raises(_lib.NedyError):
        win.G.download(_lib.RET, 0, 41 * 42 // 2)
    for s in (full, win):
        s.ctx.close()
