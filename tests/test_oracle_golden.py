"""Pin the CPU oracle to the reference's own known answers.

* calculus weights vs tests/data/calccoeff.h5 (reference tests/integration-test.cpp:5-69);
* the history integrals vs tests/integrals-test.cpp:8-212 (energy_conv, CTV1,
  Ctv_tstp, Cles2_tstp, Cles3_tstp) on the analytic fixtures of tests/set_up_g.h.
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from nedyson_b200.greens import HostGF
from fixtures import set_up_G, set_up_G_herm

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_calculus_weights_match_reference_h5():
    ref = _load("calccoeff.json")
    k = 5
    t = po.integrator_tables(k)
    # The stored interpolation table carries double-precision rounding of about
    # 1e-13 (e.g. entry (1,0) is -2.283333333333342, exactly -137/60); the tables
    # here are built in long double like src/integration.cpp:8-26 and are exact
    # to the last bit (checked below), so the norm of the difference is 1.8e-13.
    assert np.linalg.norm(np.array(ref["PInterp"]) - t["poly_interp"]) < 2.5e-13
    import mpmath
    mpmath.mp.dps = 40
    inv = mpmath.matrix([[mpmath.mpf(i) ** n for n in range(6)] for i in range(6)]) ** -1
    exact = np.array([float(inv[i, j]) for i in range(6) for j in range(6)])
    assert np.array_equal(exact, t["poly_interp"])
    assert np.linalg.norm(np.array(ref["PDiff"]) - t["poly_diff"]) < 1e-12
    assert np.linalg.norm(np.array(ref["PInteg"]) - t["poly_integ"]) < 1e-12
    assert np.linalg.norm(np.array(ref["BD"]) - t["bd"]) < 1e-12
    start = np.array([[po.gregory_weight(k, i, j) for j in range(6)] for i in range(6)]).ravel()
    assert np.linalg.norm(np.array(ref["Start"]) - start) < 1e-12
    sig = np.array([po.gregory_weight(k, i, j) for i in range(6, 12) for j in range(i + 1)])
    assert np.linalg.norm(np.array(ref["Sigma"]) - sig) < 1e-12
    om = t["Omega"].reshape(6, 6)[5]
    assert np.linalg.norm(np.array(ref["w"]) - om) < 1e-12


def test_gregory_weights_integrate_polynomials():
    # sum_j w(n,j) j^p = n^{p+1}/(p+1) for p <= k (Gregory quadrature is exact there)
    k = 5
    for n in [3, 7, 12, 40]:
        for p in range(k + 1):
            s = sum(po.gregory_weight(k, n, j) * float(j) ** p for j in range(max(n, k) + 1))
            assert abs(s - n ** (p + 1) / (p + 1)) < 1e-9 * max(1, n ** (p + 1))


@pytest.mark.parametrize("ntau", [5, 30, 64, 256])
def test_lgl_nodes(ntau):
    x, w = po.colloc_nodes(ntau)
    assert x[0] == -1.0 and x[-1] == 1.0
    assert np.allclose(x, -x[::-1], atol=0)
    assert np.all(np.diff(x) > 0)
    assert abs(w.sum() - 2.0) < 1e-13
    # exact for polynomials of degree <= 2*ntau - 1
    for p in [0, 2, 2 * ntau - 2]:
        assert abs((w * x ** p).sum() - 2.0 / (p + 1)) < 1e-12


@pytest.fixture(scope="module")
def integ():
    g = _load("integrals.json")
    Nt, Ntau, Nao, beta, dt, k = g["Nt"], g["Ntau"], g["Nao"], g["beta"], g["dt"], g["k"]
    dy = po.Dyson(Nt, Ntau, Nao, k)
    x, _ = po.colloc_nodes(Ntau)
    return g, dy, x


def _fresh(g, x):
    Nt, Ntau, Nao, beta, dt = g["Nt"], g["Ntau"], g["Nao"], g["beta"], g["dt"]
    G, Gcc, S, Scc = (HostGF(Nt, Ntau, Nao, -1) for _ in range(4))
    set_up_G(x, G, Gcc, S, Scc, dt, beta)
    return G, Gcc, S, Scc


def test_energy_conv_golden(integ):
    g, dy, x = integ
    S = HostGF(g["Nt"], g["Ntau"], g["Nao"], -1)
    G = HostGF(g["Nt"], g["Ntau"], g["Nao"], -1)
    set_up_G_herm(x, G, S, g["dt"], g["beta"])
    cases = g["cases"]["Energy Integral"]
    assert len(cases) == 7
    for c in cases:
        e = dy.energy_conv(c["t"], S, G, g["beta"], g["dt"])
        assert abs(e - c["value"][0]) < c["tol"], (c, e)


def test_ctv1_golden(integ):
    g, dy, x = integ
    G, Gcc, S, Scc = _fresh(g, x)
    cases = g["cases"]["CTV1"]
    assert len(cases) == 6
    for c in cases:
        r = dy.ctv1(S, Scc, G, c["t"], g["dt"])
        assert abs(r.sum() - complex(*c["value"])) < c["tol"], (c, r.sum())


def test_ctv_tstp_golden(integ):
    g, dy, x = integ
    cases = g["cases"]["Ctv_tstp"]
    assert len(cases) == 6
    for c in cases:
        G, Gcc, S, Scc = _fresh(g, x)
        dy.ctv_tstp(c["t"], G, G, Gcc, S, Scc, g["beta"], g["dt"])
        s = G.tv[c["t"]].sum()
        assert abs(s - complex(*c["value"])) < c["tol"], (c, s)


def test_cles2_golden(integ):
    g, dy, x = integ
    G, Gcc, S, Scc = _fresh(g, x)
    cases = g["cases"]["Cles2_tstp"]
    assert len(cases) == 6
    for c in cases:
        r = dy.cles2(G, Gcc, S, Scc, c["t"], g["dt"])
        s = r[:c["nsum"]].sum()
        assert abs(s - complex(*c["value"])) < c["tol"], (c, s)


def test_cles3_golden(integ):
    g, dy, x = integ
    G, Gcc, S, Scc = _fresh(g, x)
    cases = g["cases"]["Cles3_tstp"]
    assert len(cases) == 6
    for c in cases:
        r = dy.cles3(S, Scc, G, Gcc, c["t"], g["beta"])
        s = r[:c["nsum"]].sum()
        assert abs(s - complex(*c["value"])) < c["tol"], (c, s)
