"""Oracle self-consistency, ported from the reference's unit tests.

* GEMM chain == brute-force loop for the GF2 self-energy in its three forms
  (reference tests/mol2bSolver-test.cpp:5-265, ||diff|| < 1e-10, nao=2,
  naux=3, nt=4, ntau=5, random V and G);
* HF GEMM form == brute-force loop (reference tests/molHFSolver-test.cpp).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from nedyson_b200.greens import HostGF


def rand_gf(rng, nt, ntau, nao):
    g = HostGF(nt, ntau, nao, -1)
    for a in (g.les, g.ret, g.tv):
        a[:] = rng.uniform(-1, 1, a.shape) + 1j * rng.uniform(-1, 1, a.shape)
    return g


def rand_V(rng, nao, naux):
    return rng.uniform(-1, 1, (nao, nao, naux))


def diff(a, b):
    return max(np.linalg.norm(a.les - b.les), np.linalg.norm(a.ret - b.ret), np.linalg.norm(a.tv - b.tv))


@pytest.mark.parametrize("seed", [0, 1])
def test_df_chain_equals_loop(seed):
    rng = np.random.default_rng(seed)
    nao, naux, nt, ntau = 2, 3, 4, 5
    V = rand_V(rng, nao, naux)
    G = rand_gf(rng, nt, ntau, nao)
    S1 = HostGF(nt, ntau, nao, -1)
    S2 = HostGF(nt, ntau, nao, -1)
    s = po.DF(V)
    for t in range(nt + 1):
        s.solve(t, S1, G)
        s.solve_loop(t, S2, G)
    assert diff(S1, S2) < 1e-10
    assert np.linalg.norm(S1.les) > 1e-3


def test_df_spin_chain_equals_loop():
    rng = np.random.default_rng(7)
    nao, naux, nt, ntau = 2, 3, 4, 5
    V = rand_V(rng, nao, naux)
    G = [rand_gf(rng, nt, ntau, nao) for _ in range(2)]
    S1 = [HostGF(nt, ntau, nao, -1) for _ in range(2)]
    S2 = [HostGF(nt, ntau, nao, -1) for _ in range(2)]
    s = po.DF(V)
    for t in range(nt + 1):
        s.solve_spin(t, S1, G)
        s.solve_spin_loop(t, S2, G)
    for a, b in zip(S1, S2):
        assert diff(a, b) < 1e-10


def test_df_spin_reduces_to_restricted():
    # identical spins: unrestricted bubble sums both spins (x2), exchange per spin (x1)
    rng = np.random.default_rng(3)
    nao, naux, nt, ntau = 3, 4, 3, 4
    V = rand_V(rng, nao, naux)
    G = rand_gf(rng, nt, ntau, nao)
    S = HostGF(nt, ntau, nao, -1)
    Su = [HostGF(nt, ntau, nao, -1) for _ in range(2)]
    s = po.DF(V)
    for t in range(nt + 1):
        s.solve(t, S, G)
        s.solve_spin(t, Su, [G, G.copy()])
    assert diff(S, Su[0]) < 1e-10 and diff(S, Su[1]) < 1e-10


def test_full_chain_equals_loop():
    rng = np.random.default_rng(11)
    nao, nt, ntau = 2, 4, 5
    U = rng.uniform(-1, 1, (nao,) * 4)
    # Uexch(j,l,n,q) = 2 U(j,n,l,q) - U(j,l,n,q)   (tests/mol2bSolver-test.cpp:229-237)
    Uex = 2 * U.transpose(0, 2, 1, 3) - U
    G = rand_gf(rng, nt, ntau, nao)
    S1 = HostGF(nt, ntau, nao, -1)
    S2 = HostGF(nt, ntau, nao, -1)
    s = po.Full(U, Uex)
    for t in range(nt + 1):
        s.solve(t, S1, G)
        s.solve_loop(t, S2, G)
    assert diff(S1, S2) < 1e-10


def test_full_equals_df_when_U_is_factorised():
    # U_ijkl = sum_Q B^Q_ij B^Q_kl with symmetric B^Q makes the full-U and
    # density-fitted solvers identical
    rng = np.random.default_rng(5)
    nao, naux, nt, ntau = 3, 4, 3, 4
    V = rand_V(rng, nao, naux)
    V = 0.5 * (V + V.transpose(1, 0, 2))
    U = np.einsum("ija,kla->ijkl", V, V)
    Uex = 2 * U.transpose(0, 2, 1, 3) - U
    G = rand_gf(rng, nt, ntau, nao)
    S1 = HostGF(nt, ntau, nao, -1)
    S2 = HostGF(nt, ntau, nao, -1)
    for t in range(nt + 1):
        po.Full(U, Uex).solve(t, S1, G)
        po.DF(V).solve(t, S2, G)
    assert diff(S1, S2) < 1e-10


def test_hf_forms_equal_loops():
    rng = np.random.default_rng(2)
    nao, naux = 3, 5
    V = rand_V(rng, nao, naux)
    rho = rng.uniform(-1, 1, (nao, nao)) + 1j * rng.uniform(-1, 1, (nao, nao))
    s = po.DF(V)
    h1 = rng.uniform(-1, 1, (nao, nao)) + 0j
    h2 = h1.copy()
    s.hf(h1, rho)
    s.hf_loop(h2, rho)
    assert np.linalg.norm(h1 - h2) < 1e-10
    rho2 = rng.uniform(-1, 1, (2, nao, nao)) + 1j * rng.uniform(-1, 1, (2, nao, nao))
    hu1, hd1 = np.zeros((nao, nao), complex), np.zeros((nao, nao), complex)
    hu2, hd2 = hu1.copy(), hd1.copy()
    s.hf_spin(hu1, hd1, rho2)
    s.hf_spin_loop(hu2, hd2, rho2)
    assert np.linalg.norm(hu1 - hu2) < 1e-10 and np.linalg.norm(hd1 - hd2) < 1e-10
    U = rng.uniform(-1, 1, (nao,) * 4)
    f = po.Full(U, U)
    g1 = np.zeros((nao, nao), complex)
    g2 = g1.copy()
    f.hf(g1, rho)
    f.hf_loop(g2, rho)
    assert np.linalg.norm(g1 - g2) < 1e-10


def test_uhf_fock_matches_oracle_hf_spin():
    from nedyson_b200.inputs import make_problem, uhf_fock
    p = make_problem(5, 9, seed=41, spin=True)
    rng = np.random.default_rng(3)
    rho = []
    for _ in range(2):
        x = rng.standard_normal((5, 5)) + 1j * rng.standard_normal((5, 5))
        rho.append(0.5 * (x + x.conj().T))
    Fu, Fd = uhf_fock(p, rho[0], rho[1])
    hu, hd = p.h0.astype(complex), p.h0_dn.astype(complex)
    po.DF(p.Vija).hf_spin(hu, hd, np.stack(rho))
    assert np.abs(Fu - hu).max() < 1e-12 and np.abs(Fd - hd).max() < 1e-12


def test_uhf_equilibrium_with_equal_spins_is_rhf():
    from nedyson_b200.inputs import make_problem, uhf_equilibrium, hf_equilibrium
    p = make_problem(8, 16, seed=43, spin=True)
    q = make_problem(8, 16, seed=43)
    assert np.array_equal(p.h0, q.h0) and np.array_equal(p.Vija, q.Vija)
    p.h0_dn = p.h0.copy()
    (Fu, Fd), (mu_u, mu_d) = uhf_equilibrium(p, 10.0)
    F, mu = hf_equilibrium(q, 10.0)
    assert np.abs(Fu - F).max() < 1e-10 and np.abs(Fd - F).max() < 1e-10
    assert abs(mu_u - mu) < 1e-10 and abs(mu_d - mu) < 1e-10


def test_row_in_parts_equals_whole_row():
    """The job-range solves (used to time the CPU iteration in bounded parts) compute exactly the
    slices of the whole-row solve."""
    from nedyson_b200.greens import HostGF
    rng = np.random.default_rng(77)
    nao, naux, nt, ntau = 4, 7, 5, 6
    V = rng.uniform(-1, 1, (nao, nao, naux))
    df = po.DF(V)
    G = []
    for _ in range(2):
        g = HostGF(nt, ntau, nao, -1)
        for a in (g.les, g.ret, g.tv, g.mat):
            a[:] = rng.uniform(-1, 1, a.shape) + 1j * rng.uniform(-1, 1, a.shape)
        G.append(g)
    T = 4
    njobs = 2 * (T + 1) + ntau + 1
    whole = [HostGF(nt, ntau, nao, -1) for _ in range(2)]
    parts = [HostGF(nt, ntau, nao, -1) for _ in range(2)]
    df.solve_spin(T, whole, G)
    for lo, hi in ((0, 3), (3, 11), (11, njobs)):
        df.solve_spin_jobs(T, parts, G, lo, hi)
    for a, b in zip(parts, whole):
        for comp in ("les", "ret", "tv"):
            assert np.array_equal(getattr(a, comp), getattr(b, comp)), comp
    w1, p1 = HostGF(nt, ntau, nao, -1), HostGF(nt, ntau, nao, -1)
    df.solve(T, w1, G[0])
    df.solve_jobs(T, p1, G[0], 0, 5)
    df.solve_jobs(T, p1, G[0], 5, njobs)
    for comp in ("les", "ret", "tv"):
        assert np.array_equal(getattr(p1, comp), getattr(w1, comp)), comp
