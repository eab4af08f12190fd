"""Oracle checks of the Dyson machinery that need no GPU.

* the numpy free Green's function (product host setup) equals the oracle's
  G0_from_h0 (reference src/dyson_free.h:226-297);
* with Sigma = 0 the Dyson step propagates the free Green's function: the
  retarded, mixed and lesser rows stay on the exact free solution up to the
  order-k BDF/Gregory error;
* the bootstrap of a free (TTI) start is already converged;
* a short interacting run keeps G^<(t,t) Hermitian-consistent and particle
  number conserved (no drive).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from nedyson_b200.greens import HostGF
from nedyson_b200.inputs import make_problem, g0_from_h0, hf_equilibrium
from simref import OracleDecompSim


def test_g0_numpy_equals_oracle():
    p = make_problem(4, 6, seed=3)
    nt, ntau, beta, dt, k = 8, 16, 5.0, 0.05, 5
    F, mu = hf_equilibrium(p, beta)
    x, _ = po.colloc_nodes(ntau)
    a = HostGF(nt, ntau, 4, -1)
    b = HostGF(nt, ntau, 4, -1)
    g0_from_h0(a, x, mu, F, beta, dt, k)
    dy = po.Dyson(nt, ntau, 4, k)
    dy.g0_from_h0(b, mu, F, beta, dt)
    b.mat[:] = a.mat  # the constant-h oracle routine leaves G^M to the caller (dyson_free.h:248-256)
    for comp in ("les", "ret", "tv"):
        assert np.abs(getattr(a, comp) - getattr(b, comp)).max() < 1e-12, comp


def test_free_propagation():
    p = make_problem(3, 4, seed=1)
    nt, ntau, beta, dt, k = 30, 24, 4.0, 0.02, 5
    F, mu = hf_equilibrium(p, beta)
    x, _ = po.colloc_nodes(ntau)
    exact = HostGF(nt, ntau, 3, -1)
    g0_from_h0(exact, x, mu, F, beta, dt, nt)  # exact free G on the whole [0,nt]^2
    G = HostGF(nt, ntau, 3, -1)
    g0_from_h0(G, x, mu, F, beta, dt, k)
    S = HostGF(nt, ntau, 3, -1)
    hmf = np.repeat(F[None].astype(complex), nt + 1, axis=0)
    dy = po.Dyson(nt, ntau, 3, k)
    err = dy.dyson_start(G, S, hmf, mu, beta, dt)
    assert err < 1e-8
    for t in range(k + 1, nt + 1):
        dy.extrapolate(t, G)
        dy.dyson_step(t, G, S, hmf, mu, beta, dt)
    for t in (k + 1, nt // 2, nt):
        assert np.abs(G.ret_row(t) - exact.ret_row(t)).max() < 1e-8
        assert np.abs(G.les_col(t) - exact.les_col(t)).max() < 1e-8
        assert np.abs(G.tv[t] - exact.tv[t]).max() < 1e-8


def test_interacting_run_conserves_particles():
    p = make_problem(4, 8, seed=5)
    sim = OracleDecompSim(p, nt=12, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=3)
    sim.free_gf()
    sim.do_boot(max_iter=20)
    n0 = np.trace(sim.G.get_dm(0)).real
    for t in range(6, 13):
        sim.do_tstp(t)
    n1 = np.trace(sim.G.get_dm(12)).real
    assert abs(n1 - n0) < 1e-6
    rho = sim.G.get_dm(12)
    assert np.abs(rho - rho.conj().T).max() < 1e-8


def test_unrestricted_run_conserves_particles_per_spin():
    """Unrestricted oracle driver (DecompSpinSimulation restated): each spin's particle
    number is conserved through the bootstrap and a driven run, and the two spins, with
    their own h0, evolve differently."""
    from simref import OracleDecompSpinSim
    p = make_problem(4, 8, seed=9, spin=True)
    sim = OracleDecompSpinSim(p, nt=12, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=3, drive_kind="gauss",
                              drive_kw=dict(E0=0.5, t0=0.2, sigma=0.05))
    sim.free_gf()
    sim.do_boot(max_iter=20)
    n0 = [np.trace(sim.G[s].get_dm(0)).real for s in range(2)]
    for t in range(6, 13):
        sim.do_tstp(t)
    for s in range(2):
        rho = sim.G[s].get_dm(12)
        assert abs(np.trace(rho).real - n0[s]) < 1e-6
        assert np.abs(rho - rho.conj().T).max() < 1e-8
    assert np.abs(sim.G[0].get_dm(12) - sim.G[1].get_dm(12)).max() > 1e-3
