"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 path tolerance: max |GPU - oracle| <= 1e-10 * max(1, max |oracle|) per
component, on seeded inputs (the reference's own loop-vs-GEMM tests use 1e-10).
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from nedyson_b200 import api
from nedyson_b200.greens import HostGF
from nedyson_b200.inputs import make_problem, g0_from_h0, hf_equilibrium
from nedyson_b200.simulation import DecompSimulation
from fixtures import set_up_G_herm
from simref import OracleDecompSim

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def rand_gf(rng, nt, ntau, nao, scale=1.0):
    g = HostGF(nt, ntau, nao, -1)
    for a in (g.les, g.ret, g.tv, g.mat):
        a[:] = scale * (rng.uniform(-1, 1, a.shape) + 1j * rng.uniform(-1, 1, a.shape))
    return g


def cmp_gf(a: HostGF, b: HostGF, tol=TOL, rows=None):
    for comp in ("les", "ret", "tv"):
        x, y = getattr(a, comp), getattr(b, comp)
        assert rel(x, y) < tol, (comp, rel(x, y))


@pytest.mark.parametrize("nao,naux,nt,ntau", [(2, 3, 4, 5), (4, 6, 6, 7), (7, 11, 3, 4), (32, 64, 2, 4)])
def test_sigma_decomp(nao, naux, nt, ntau):
    rng = np.random.default_rng(nao * 100 + naux)
    V = rng.uniform(-1, 1, (nao, nao, naux))
    G = rand_gf(rng, nt, ntau, nao)
    So = HostGF(nt, ntau, nao, -1)
    df = po.DF(V)
    ctx = api.Context(max(nt, 5), ntau, nao, 5, 1.0, 0.01)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    Sd = api.green_func(ctx, nt, ntau, nao, -1)
    s = api.molGF2SolverDecomp(ctx, V)
    for t in range(nt + 1):
        df.solve(t, So, G)
        s.solve(t, Sd, Gd)
    cmp_gf(Sd.to_host(), So, 1e-12)


@pytest.mark.parametrize("nspin", [1, 2])
def test_sigma_decomp_symmetric_BQ(nspin):
    # real symmetric B^Q selects the retarded row Sigma^R = Sigma^>(T,t) + Sigma^<(t,T)^+
    nao, naux, nt, ntau = 6, 9, 5, 6
    p = make_problem(nao, naux, seed=40 + nspin)
    rng = np.random.default_rng(5)
    G = [rand_gf(rng, nt, ntau, nao) for _ in range(nspin)]
    So = [HostGF(nt, ntau, nao, -1) for _ in range(nspin)]
    ctx = api.Context(max(nt, 5), ntau, nao, 5, 1.0, 0.01)
    Gd = [api.green_func(ctx, nt, ntau, nao, -1).from_host(g) for g in G]
    Sd = [api.green_func(ctx, nt, ntau, nao, -1) for _ in range(nspin)]
    df = po.DF(p.Vija)
    if nspin == 1:
        s = api.molGF2SolverDecomp(ctx, p.Vija)
        for t in range(nt + 1):
            df.solve(t, So[0], G[0])
            s.solve(t, Sd[0], Gd[0])
    else:
        s = api.molGF2SolverSpinDecomp(ctx, p.Vija)
        for t in range(nt + 1):
            df.solve_spin(t, So, G)
            s.solve(t, Sd, Gd)
    for a, b in zip(Sd, So):
        cmp_gf(a.to_host(), b, 1e-12)


def test_sigma_decomp_chunked_workspace():
    # a small workspace budget forces several slice chunks and exchange sub-chunks
    rng = np.random.default_rng(9)
    nao, naux, nt, ntau = 8, 12, 9, 10
    V = rng.uniform(-1, 1, (nao, nao, naux))
    G = rand_gf(rng, nt, ntau, nao)
    So = HostGF(nt, ntau, nao, -1)
    ctx = api.Context(nt, ntau, nao, 5, 1.0, 0.01, workspace_bytes=200_000)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    Sd = api.green_func(ctx, nt, ntau, nao, -1)
    s = api.molGF2SolverDecomp(ctx, V)
    df = po.DF(V)
    for t in (0, 5, nt):
        df.solve(t, So, G)
        s.solve(t, Sd, Gd)
    cmp_gf(Sd.to_host(), So, 1e-12)


def test_sigma_spin_decomp():
    rng = np.random.default_rng(21)
    nao, naux, nt, ntau = 4, 5, 5, 6
    V = rng.uniform(-1, 1, (nao, nao, naux))
    G = [rand_gf(rng, nt, ntau, nao) for _ in range(2)]
    So = [HostGF(nt, ntau, nao, -1) for _ in range(2)]
    ctx = api.Context(nt, ntau, nao, 5, 1.0, 0.01)
    Gd = [api.green_func(ctx, nt, ntau, nao, -1).from_host(g) for g in G]
    Sd = [api.green_func(ctx, nt, ntau, nao, -1) for _ in range(2)]
    s = api.molGF2SolverSpinDecomp(ctx, V)
    df = po.DF(V)
    for t in range(nt + 1):
        df.solve_spin(t, So, G)
        s.solve(t, Sd, Gd)
    for a, b in zip(Sd, So):
        cmp_gf(a.to_host(), b, 1e-12)


def test_sigma_full():
    rng = np.random.default_rng(4)
    nao, nt, ntau = 4, 6, 8
    U = rng.uniform(-1, 1, (nao,) * 4)
    Uex = 2 * U.transpose(0, 2, 1, 3) - U
    G = rand_gf(rng, nt, ntau, nao)
    So = HostGF(nt, ntau, nao, -1)
    ctx = api.Context(nt, ntau, nao, 5, 1.0, 0.01)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    Sd = api.green_func(ctx, nt, ntau, nao, -1)
    s = api.molGF2Solver(ctx, U, Uex)
    f = po.Full(U, Uex)
    for t in range(nt + 1):
        f.solve(t, So, G)
        s.solve(t, Sd, Gd)
    cmp_gf(Sd.to_host(), So, 1e-12)


def test_hf_variants():
    rng = np.random.default_rng(8)
    nao, naux, nt = 6, 10, 6
    V = rng.uniform(-1, 1, (nao, nao, naux))
    rho = rng.uniform(-1, 1, (nao, nao)) + 1j * rng.uniform(-1, 1, (nao, nao))
    ctx = api.Context(nt, 8, nao, 5, 1.0, 0.01)
    h0 = rng.uniform(-1, 1, (nt + 1, nao, nao)) + 0j
    hm = api.hmf_buffer(ctx, nao, h0)
    rb = api.DeviceBuffer.from_array(ctx, rho)
    s = api.molGF2SolverDecomp(ctx, V)
    s.solve_HF(3, hm, rb)
    out = hm.download((nt + 1, nao, nao))
    ref = h0.copy()
    po.DF(V).hf(ref[3], rho)
    assert rel(out, ref) < 1e-13
    # spin
    rho2 = rng.uniform(-1, 1, (2, nao, nao)) + 1j * rng.uniform(-1, 1, (2, nao, nao))
    hu, hd = api.hmf_buffer(ctx, nao, h0), api.hmf_buffer(ctx, nao, h0)
    sp = api.molGF2SolverSpinDecomp(ctx, V)
    sp.solve_HF(2, [hu, hd], api.DeviceBuffer.from_array(ctx, rho2))
    ru, rd = h0.copy(), h0.copy()
    po.DF(V).hf_spin(ru[2], rd[2], rho2)
    assert rel(hu.download(ru.shape), ru) < 1e-13 and rel(hd.download(rd.shape), rd) < 1e-13
    # full U
    U = rng.uniform(-1, 1, (nao,) * 4)
    hf = api.hmf_buffer(ctx, nao, h0)
    api.molGF2Solver(ctx, U, U).solve_HF(1, hf, rb)
    rf = h0.copy()
    po.Full(U, U).hf(rf[1], rho)
    assert rel(hf.download(rf.shape), rf) < 1e-13


def test_extrapolate():
    rng = np.random.default_rng(12)
    nao, nt, ntau, k = 3, 14, 6, 5
    G = rand_gf(rng, nt, ntau, nao)
    ctx = api.Context(nt, ntau, nao, k, 1.0, 0.01)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    dy = po.Dyson(nt, ntau, nao, k)
    for n in (k + 1, k + 3, 11, nt):
        dy.extrapolate(n, G)
        api.dyson(ctx).Extrapolate(n, Gd)
    cmp_gf(Gd.to_host(), G, 1e-13)


def _state(nao, naux, nt, ntau, beta, dt, k, seed, sigma_scale=0.05):
    """Free (HF) G on [0, nt], random small Sigma history, random Hermitian hmf."""
    p = make_problem(nao, naux, seed)
    F, mu = hf_equilibrium(p, beta)
    x, _ = po.colloc_nodes(ntau)
    G = HostGF(nt, ntau, nao, -1)
    g0_from_h0(G, x, mu, F, beta, dt, nt)
    rng = np.random.default_rng(seed + 1)
    S = rand_gf(rng, nt, ntau, nao, sigma_scale)
    hmf = np.zeros((nt + 1, nao, nao), complex)
    for t in range(nt + 1):
        a = rng.normal(size=(nao, nao)) * 0.05
        hmf[t] = F + 0.5 * (a + a.T)
    return p, G, S, hmf, mu


@pytest.mark.parametrize("nao,T", [(3, 6), (3, 9), (5, 14), (16, 20), (32, 8)])
def test_dyson_step(nao, T):
    nt, ntau, beta, dt, k = max(T, 12), 12, 4.0, 0.02, 5
    p, G, S, hmf, mu = _state(nao, 4, nt, ntau, beta, dt, k, seed=nao + T)
    ctx = api.Context(nt, ntau, nao, k, beta, dt)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    Sd = api.green_func(ctx, nt, ntau, nao, -1).from_host(S)
    hb = api.hmf_buffer(ctx, nao, hmf)
    dy = po.Dyson(nt, ntau, nao, k)
    eo, parts_o = dy.dyson_step(T, G, S, hmf, mu, beta, dt)
    eg, parts_g = api.dyson(ctx).dyson_step(T, Gd, Sd, hb, mu)
    Gh = Gd.to_host()
    assert rel(Gh.ret_row(T), G.ret_row(T)) < TOL
    assert rel(Gh.tv[T], G.tv[T]) < TOL
    assert rel(Gh.les_col(T), G.les_col(T)) < TOL
    assert abs(eg - eo) <= 1e-8 * max(1.0, abs(eo))


@pytest.mark.parametrize("nao", [4, 32])
def test_dyson_start(nao):
    nt, ntau, beta, dt, k = 10, 14, 5.0, 0.02, 5
    p, G, S, hmf, mu = _state(nao, 4, nt, ntau, beta, dt, k, seed=31)
    ctx = api.Context(nt, ntau, nao, k, beta, dt)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    Sd = api.green_func(ctx, nt, ntau, nao, -1).from_host(S)
    hb = api.hmf_buffer(ctx, nao, hmf)
    eo = po.Dyson(nt, ntau, nao, k).dyson_start(G, S, hmf, mu, beta, dt)
    eg = api.dyson(ctx).dyson_start(Gd, Sd, hb, mu)
    cmp_gf(Gd.to_host(), G)
    assert abs(eg - eo) <= 1e-8 * max(1.0, abs(eo))


def test_energy_conv_golden_on_gpu():
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "integrals.json")))
    Nt, Ntau, Nao, beta, dt = gold["Nt"], gold["Ntau"], gold["Nao"], gold["beta"], gold["dt"]
    x, _ = po.colloc_nodes(Ntau)
    S = HostGF(Nt, Ntau, Nao, -1)
    G = HostGF(Nt, Ntau, Nao, -1)
    set_up_G_herm(x, G, S, dt, beta)
    ctx = api.Context(Nt, Ntau, Nao, 5, beta, dt)
    Gd = api.green_func(ctx, Nt, Ntau, Nao, -1).from_host(G)
    Sd = api.green_func(ctx, Nt, Ntau, Nao, -1).from_host(S)
    for c in gold["cases"]["Energy Integral"]:
        e = api.dyson(ctx).energy_conv(c["t"], Sd, Gd)
        assert abs(e - c["value"][0]) < c["tol"], (c, e)


@pytest.mark.parametrize("drive_kind", ["none", "gauss"])
def test_simulation_matches_oracle(drive_kind):
    p = make_problem(4, 8, seed=17)
    kw = dict(nt=14, ntau=16, beta=5.0, dt=0.02, k=5, corr_steps=2, drive_kind=drive_kind,
              drive_kw=dict(E0=0.5, t0=0.2, sigma=0.05))
    ref = OracleDecompSim(p, **kw)
    ref.free_gf()
    ref.do_boot(max_iter=10)
    gpu = DecompSimulation(p, **kw)
    gpu.free_gf()
    gpu.do_boot(max_iter=10)
    cmp_gf(gpu.G.to_host(), ref.G)
    for t in range(6, 15):
        ref.do_tstp(t)
        gpu.do_tstp(t)
    cmp_gf(gpu.G.to_host(), ref.G)
    cmp_gf(gpu.Sigma.to_host(), ref.S)


# Split-precision self-energy (BF16 pieces on tcgen05, FP32 accumulation): the
# contractions carry a relative error of a few 1e-6 of the largest element with
# three pieces per operand, a few 1e-5 with two; the bounds below are stated per
# component against the FP64 oracle.
SPLIT_TOL = {"bf16x3": 5e-5, "bf16x2": 5e-4}


@pytest.mark.parametrize("mode", ["bf16x3", "bf16x2"])
@pytest.mark.parametrize("nao,naux,sym,nspin", [(16, 48, True, 1), (16, 40, False, 1), (12, 36, True, 2),
                                                (23, 70, False, 1), (13, 40, True, 2)])
def test_sigma_split(nao, naux, sym, nspin, mode):
    from nedyson_b200 import _lib
    prec = {"bf16x3": _lib.PREC_SPLIT_BF16X3, "bf16x2": _lib.PREC_SPLIT_BF16X2}[mode]
    rng = np.random.default_rng(700 + nao + naux)
    V = rng.uniform(-1, 1, (nao, nao, naux)) / np.sqrt(naux)
    if sym:
        V = 0.5 * (V + V.transpose(1, 0, 2))
    nt, ntau = 4, 6
    Gs = [rand_gf(rng, nt, ntau, nao) for _ in range(nspin)]
    So = [HostGF(nt, ntau, nao, -1) for _ in range(nspin)]
    ctx = api.Context(max(nt, 5), ntau, nao, 5, 1.0, 0.01)
    ctx.set_precision(prec)
    Gd = [api.green_func(ctx, nt, ntau, nao, -1).from_host(g) for g in Gs]
    Sd = [api.green_func(ctx, nt, ntau, nao, -1) for _ in range(nspin)]
    if nspin == 1:
        df, s = po.DF(V), api.molGF2SolverDecomp(ctx, V)
        for t in range(nt + 1):
            df.solve(t, So[0], Gs[0])
            s.solve(t, Sd[0], Gd[0])
    else:
        df, s = po.DF(V), api.molGF2SolverSpinDecomp(ctx, V)
        for t in range(nt + 1):
            df.solve_spin(t, So, Gs)
            s.solve(t, Sd, Gd)
    for sp in range(nspin):
        got = Sd[sp].to_host()
        for comp in ("les", "ret", "tv"):
            x, y = getattr(got, comp), getattr(So[sp], comp)
            err = np.abs(x - y).max() / np.abs(y).max()
            print(f"split {mode} nao={nao} naux={naux} nspin={nspin} {comp}: {err:.3e}")
            assert err < SPLIT_TOL[mode], (comp, err)
            assert err > 0.0  # the split path ran, not the FP64 one
