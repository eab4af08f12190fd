"""CPU restatement of the equilibrium (Matsubara) GF2 state on the collocation grid
(test infrastructure only: tests and the CPU checks import it, the library does not).

The reference obtains this state from the external gfmol solver (call sites
src/molNEsim_decomp_impl.h:23-33, :45, :51; L_to_Tau :146-167), which is not part of
the reference tree, so this is a restatement of the equations, not of gfmol's code:

    Sigma^M[G^M]  the density-fitted GF2 self-energy of the t = 0 mixed row
                  (mol2bSolver_decomp_impl.h:412-429 through oracle/sigma.cpp), with
                  G^tv(0, tau) = -i G^M(beta - tau) and Sigma^M(tau) = i Sigma^tv(0, beta - tau);
    F             h0 + HF(rho), rho = -G^M(beta)            (molHFSolver.cpp:81-110);
    Dyson         G = G_ref + G_ref * (F - F_ref + Sigma^M) * G on the degree-ntau
                  interpolants, (A * B)(tau_m) = sum_i K_A[m][i] B_i with K_A the
                  mixing kernel (oracle/collocation.cpp) of B(x) = A(-x).

Unlike the engine, which relaxes G by fixed-point sweeps, every outer iteration here solves
the linear Dyson equation for G exactly (one dense solve of size (ntau+1) nao), so the two
reach the common fixed point by different routes.
"""
from __future__ import annotations

import numpy as np

from . import pyoracle as po


def _mirror(A, s):
    """s * A[ntau - j] for every node j."""
    return s * A[::-1]


def sigma_mat(df: po.DF, Gmat, beta, spin=False):
    """Sigma^M of G^M (list of (np, N, N) arrays, one per spin)."""
    from nedyson_b200.greens import HostGF
    ns = len(Gmat)
    np1, N, _ = Gmat[0].shape
    G, S = [], []
    for s in range(ns):
        g = HostGF(0, np1 - 1, N, -1)
        g.tv[0] = _mirror(Gmat[s], -1j)
        G.append(g)
        S.append(HostGF(0, np1 - 1, N, -1))
    if ns == 2:
        df.solve_spin(0, S, G)
    else:
        df.solve(0, S[0], G[0])
    return [_mirror(S[s].tv[0], 1j) for s in range(ns)]


def conv_kernel(dy: po.Dyson, A, beta, sig=-1.0):
    """K[m][i] with (A * B)(tau_m) = sum_i K[m][i] B_i."""
    return dy.mixing_kernel(np.ascontiguousarray(_mirror(A, sig)), beta, sig)


def solve(p, beta, ntau, Fs, mus, Gref, spin=False, max_iter=200, tol=1e-12):
    """Equilibrium GF2 state from G_ref (free G^M of Fs at mus): returns (Gmat, Smat, F, iters)."""
    ns = 2 if spin else 1
    N = p.nao
    np1 = ntau + 1
    dy = po.Dyson(0, ntau, N, 5)
    df = po.DF(p.Vija)
    Kref = [conv_kernel(dy, Gref[s], beta) for s in range(ns)]
    G = [g.copy() for g in Gref]
    it = 0
    for it in range(1, max_iter + 1):
        rho = np.stack([-G[s][-1] for s in range(ns)])
        if ns == 2:
            hu, hd = p.h0_of(0).astype(complex), p.h0_of(1).astype(complex)
            df.hf_spin(hu, hd, rho)
            F = [hu, hd]
        else:
            h = p.h0.astype(complex)
            df.hf(h, rho[0])
            F = [h]
        Sm = sigma_mat(df, G, beta, spin)
        Gn = []
        for s in range(ns):
            Ks = conv_kernel(dy, Sm[s], beta)
            dF = F[s] - Fs[s]
            # G = Gref + Kref (Ks G + dF G): (I - Kref (Ks + I x dF)) G = Gref, blocks (m, i) of N x N
            Ks2 = Ks.transpose(0, 2, 1, 3).reshape(np1 * N, np1 * N)
            D = np.kron(np.eye(np1), dF)
            Kr2 = Kref[s].transpose(0, 2, 1, 3).reshape(np1 * N, np1 * N)
            A = np.eye(np1 * N) - Kr2 @ (Ks2 + D)
            x = np.linalg.solve(A, Gref[s].reshape(np1 * N, N))
            Gn.append(x.reshape(np1, N, N))
        d = max(np.abs(Gn[s] - G[s]).max() for s in range(ns))
        G = Gn
        if d <= tol:
            break
    rho = np.stack([-G[s][-1] for s in range(ns)])
    if ns == 2:
        hu, hd = p.h0_of(0).astype(complex), p.h0_of(1).astype(complex)
        df.hf_spin(hu, hd, rho)
        F = [hu, hd]
    else:
        h = p.h0.astype(complex)
        df.hf(h, rho[0])
        F = [h]
    return G, sigma_mat(df, G, beta, spin), F, it
