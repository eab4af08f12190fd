"""Equilibrium (Matsubara) GF2 state on the collocation grid (nedy_matsubara_gf2).

* GPU fixed-point solver against the CPU restatement (oracle/matsubara.py), which solves
  the linear Dyson equation of every outer iteration exactly: the same fixed point,
  restricted and unrestricted, to 1e-10;
* the physics check that pins the conventions: propagated without a drive, the GF2
  equilibrium is stationary (the density and G^R(t, t-1) stay at their t = 0 values to
  about 1e-10), while the Hartree-Fock start relaxes (drift 1e-4 in the density).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from oracle import matsubara as om
from nedyson_b200 import api
from nedyson_b200.greens import HostGF
from nedyson_b200.inputs import make_problem, hf_equilibrium, uhf_equilibrium, g0_from_h0, gf2_equilibrium
from simref import OracleDecompSim


def _oracle_eq(p, beta, ntau, spin):
    if spin:
        Fs, mus = uhf_equilibrium(p, beta)
    else:
        F, mu = hf_equilibrium(p, beta)
        Fs, mus = [F], [mu]
    x, _ = po.colloc_nodes(ntau)
    Gref = []
    for s in range(len(Fs)):
        g = HostGF(-1, ntau, p.nao, -1)
        g0_from_h0(g, x, mus[s], Fs[s], beta, 0.01, -1)
        Gref.append(g.mat.copy())
    return om.solve(p, beta, ntau, Fs, mus, Gref, spin=spin)


def test_oracle_equilibrium_is_stationary():
    """CPU: the oracle's GF2 equilibrium propagated without a drive stays put (the HF one does not)."""
    p = make_problem(4, 8, seed=3)
    beta, ntau = 10.0, 24
    G, S, F, it = _oracle_eq(p, beta, ntau, False)
    drift = {}
    for label, eq in (("HF", None), ("GF2", (F[0], G[0]))):
        sim = OracleDecompSim(p, nt=16, ntau=ntau, beta=beta, dt=0.02, k=5, corr_steps=4)
        if eq:
            sim.set_equilibrium(*eq)
        sim.free_gf()
        sim.do_boot(max_iter=40)
        rho0 = sim.G.get_dm(0)
        d = 0.0
        for t in range(6, 17):
            sim.do_tstp(t)
            d = max(d, float(np.abs(sim.G.get_dm(t) - rho0).max()))
        drift[label] = d
    assert drift["GF2"] < 1e-9 and drift["HF"] > 1e-5, drift


@pytest.mark.gpu
@pytest.mark.parametrize("spin", [False, True])
def test_matsubara_gpu_matches_oracle(spin):
    p = make_problem(5, 10, seed=8, spin=spin)
    beta, ntau = 10.0, 32
    Go, So, Fo, _ = _oracle_eq(p, beta, ntau, spin)
    ctx = api.Context(5, ntau, p.nao, 5, beta, 0.01)
    r = gf2_equilibrium(ctx, p, beta, spin=spin, tol=1e-13)
    assert r["diff"] <= 1e-13 and r["iters"] > 3
    for s in range(2 if spin else 1):
        for name, a, b in (("G^M", r["Gmat"][s], Go[s]), ("Sigma^M", r["Smat"][s], So[s]), ("F", r["F"][s], Fo[s])):
            e = float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))
            print(f"spin={spin} s={s} {name}: {e:.3e}")
            assert e < 1e-10, (s, name, e)
    ctx.close()


@pytest.mark.gpu
def test_gpu_run_from_gf2_equilibrium_is_stationary():
    from nedyson_b200.simulation import DecompSimulation
    p = make_problem(6, 12, seed=9)
    beta, ntau = 10.0, 32
    ctx = api.Context(5, ntau, p.nao, 5, beta, 0.02)
    r = gf2_equilibrium(ctx, p, beta)
    ctx.close()
    drift = {}
    for label in ("HF", "GF2"):
        sim = DecompSimulation(p, 20, ntau, beta, 0.02, corr_steps=4)
        if label == "GF2":
            sim.set_equilibrium(r["F"][0], r["Gmat"][0])
        sim.free_gf()
        sim.do_boot(max_iter=40)
        g = sim.G.to_host()
        rho0 = g.get_dm(0)
        for t in range(6, 21):
            sim.do_tstp(t)
        g = sim.G.to_host()
        drift[label] = max(float(np.abs(g.get_dm(t) - rho0).max()) for t in range(6, 21))
        sim.ctx.close()
    print("density drift over 15 steps:", drift)
    assert drift["GF2"] < 1e-9 and drift["HF"] > 1e-5, drift
