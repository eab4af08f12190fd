"""Spin-unrestricted density-fitted GF2 time stepping (reference
src/molNEsim_decomp_spin_impl.h), through the C ABI, against the CPU oracle.

Tolerances: FP64 path max |GPU - oracle| <= 1e-10 * max(1, max |oracle|) per
component; the residual-exit entry with tol = 0 runs the same iterations as the
fixed-count entry and must agree to 1e-12; the split-precision form at
tol = 1e-8 must stay within 1e-7 of the FP64 trajectory.
"""
import numpy as np
import pytest

from nedyson_b200 import _lib
from nedyson_b200.inputs import make_problem
from nedyson_b200.simulation import DecompSimulation, DecompSpinSimulation
from simref import OracleDecompSpinSim

TOL = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def cmp_gf(a, b, tol=TOL):
    for comp in ("les", "ret", "tv"):
        x, y = getattr(a, comp), getattr(b, comp)
        assert rel(x, y) < tol, (comp, rel(x, y))


KW = dict(nt=12, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=2, drive_kind="gauss",
          drive_kw=dict(E0=0.5, t0=0.2, sigma=0.05))


@pytest.mark.gpu
def test_spin_simulation_matches_oracle():
    p = make_problem(4, 8, seed=19, spin=True)
    ref = OracleDecompSpinSim(p, **KW)
    ref.free_gf()
    ref.do_boot(max_iter=10)
    gpu = DecompSpinSimulation(p, **KW)
    gpu.free_gf()
    gpu.do_boot(max_iter=10)
    for s in range(2):
        cmp_gf(gpu.G[s].to_host(), ref.G[s])
    for t in range(6, 13):
        ref.do_tstp(t)
        gpu.do_tstp(t)
    for s in range(2):
        cmp_gf(gpu.G[s].to_host(), ref.G[s])
        cmp_gf(gpu.Sigma[s].to_host(), ref.S[s])
    # the two spins really differ (independent h0 per spin)
    g0, g1 = gpu.G[0].to_host(), gpu.G[1].to_host()
    assert np.abs(g0.les - g1.les).max() > 1e-3


@pytest.mark.gpu
def test_spin_identical_spins_equal_restricted():
    p = make_problem(6, 12, seed=23, spin=True)
    p.h0_dn = p.h0.copy()
    sp = DecompSpinSimulation(p, **KW)
    rs = DecompSimulation(p, **KW)
    for sim in (sp, rs):
        sim.free_gf()
        sim.do_boot(max_iter=10)
    for t in range(6, 11):
        sp.do_tstp(t)
        rs.do_tstp(t)
    g = rs.G.to_host()
    for s in range(2):
        cmp_gf(sp.G[s].to_host(), g)


@pytest.mark.gpu
def test_spin_tol_entry_matches_fixed_iterations():
    p = make_problem(6, 12, seed=29, spin=True)
    a = DecompSpinSimulation(p, **dict(KW, corr_steps=3))
    b = DecompSpinSimulation(p, **dict(KW, corr_steps=3))
    for sim in (a, b):
        sim.free_gf()
        sim.do_boot(max_iter=10)
        for t in range(6, 9):
            sim.do_tstp(t)
    for t in range(9, 13):
        a.do_tstp(t)
        it, hist = b.do_tstp_tol(t, 0.0, 3)
        assert it == 3 and len(hist) == 3
        assert hist[2] < hist[0]  # the corrector contracts
    for s in range(2):
        cmp_gf(b.G[s].to_host(), a.G[s].to_host(), 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["bf16x3", "bf16x2"])
def test_spin_split_tol_trajectory_close_to_fp64(mode):
    p = make_problem(16, 48, seed=31, spin=True)
    kw = dict(nt=16, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=5, drive_kind="gauss",
              drive_kw=dict(E0=0.1, t0=0.2, sigma=0.05))
    a = DecompSpinSimulation(p, **kw)
    b = DecompSpinSimulation(p, **kw)
    for sim in (a, b):
        sim.free_gf()
        sim.do_boot(max_iter=20)
    b.ctx.set_precision({"bf16x3": _lib.PREC_SPLIT_BF16X3, "bf16x2": _lib.PREC_SPLIT_BF16X2}[mode])
    its = []
    for t in range(6, 17):
        a.do_tstp(t)
        it, _ = b.do_tstp_tol(t, 1e-8, 5)
        its.append(it)
    assert max(its) <= 5 and min(its) >= 1
    for s in range(2):
        ga, gb = a.G[s].to_host(), b.G[s].to_host()
        for comp in ("les", "ret", "tv"):
            d = np.abs(getattr(ga, comp) - getattr(gb, comp)).max()
            print(f"spin split {mode} spin {s} {comp}: max|dG| {d:.3e}")
            assert d < 1e-7, (s, comp, d)
