"""Seeded synthetic inputs and the equilibrium starting state.

The reference reads molecular integrals from HDF5 and obtains its equilibrium
state from the external gfmol Matsubara solver; here both come from seeded
random numbers and a Hartree-Fock equilibrium, identical for the CUDA path and
for the CPU oracle:

* h0: symmetric N(0,1) matrix, upper half of the spectrum shifted so the gap at
  half filling is >= ``gap``;
* B^Q: symmetric N(0,1) matrices scaled so that ||U||_F = ``u_norm`` with
  U_ijkl = sum_Q B^Q_ij B^Q_kl; Vija[i, j, Q] = B^Q_ij;
* D: symmetric N(0,1) dipole matrix; drives E(t) gated to exactly 0 for
  t <= k*dt (the bootstrap assumes a time-translation-invariant start,
  reference src/molNEsim.cpp:38-49);
* equilibrium: self-consistent restricted HF Fock matrix F and chemical
  potential mu at mid-gap; G^M(tau) and the first k+1 time steps of G are the
  free Green's function of F (G0_from_h0, reference src/dyson_free.h:226-297).
* spin-unrestricted problems (``make_problem(..., spin=True)``): a second,
  independent h0 for spin down, drawn after every restricted input so that the
  spin-up problem equals the restricted one of the same seed; the same B^Q and
  D for both spins; the equilibrium is the unrestricted HF one, with its own
  Fock matrix and mid-gap mu per spin.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .greens import HostGF


@dataclass
class Problem:
    nao: int
    naux: int
    h0: np.ndarray
    Vija: np.ndarray
    D: np.ndarray
    seed: int
    meta: dict = field(default_factory=dict)
    h0_dn: np.ndarray | None = None   # spin-down one-body Hamiltonian (unrestricted problems)

    @property
    def spin(self) -> bool:
        return self.h0_dn is not None

    def h0_of(self, s: int) -> np.ndarray:
        return self.h0_dn if s == 1 else self.h0

    @property
    def U(self):
        return np.einsum("ija,kla->ijkl", self.Vija, self.Vija)

    @property
    def Uexch(self):
        # Uexch(j,l,n,q) = 2 U(j,n,l,q) - U(j,l,n,q)   (reference tests/mol2bSolver-test.cpp:229-237)
        U = self.U
        return 2 * U.transpose(0, 2, 1, 3) - U


def _gapped_h0(rng, nao: int, gap: float) -> np.ndarray:
    a = rng.normal(size=(nao, nao))
    h0 = 0.5 * (a + a.T)
    w, v = np.linalg.eigh(h0)
    nocc = nao // 2
    if 0 < nocc < nao:
        g = w[nocc] - w[nocc - 1]
        if g < gap:
            w[nocc:] += gap - g
    h0 = (v * w) @ v.T
    return 0.5 * (h0 + h0.T)


def make_problem(nao: int, naux: int, seed: int, gap: float = 0.5, u_norm: float = 0.5,
                 spin: bool = False) -> Problem:
    rng = np.random.default_rng(seed)
    h0 = _gapped_h0(rng, nao, gap)
    B = rng.normal(size=(naux, nao, nao))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    # ||U||_F^2 = sum_{QP} (tr B^Q B^P)^2  (B symmetric)
    gram = np.einsum("qij,pij->qp", B, B)
    nrm = math.sqrt((gram ** 2).sum())
    B *= math.sqrt(u_norm / nrm)
    Vija = np.ascontiguousarray(B.transpose(1, 2, 0))
    d = rng.normal(size=(nao, nao))
    D = 0.5 * (d + d.T)
    h0_dn = _gapped_h0(rng, nao, gap) if spin else None
    return Problem(nao, naux, h0, Vija, D, seed, h0_dn=h0_dn)


def drive(kind: str, t: float, k: int, dt: float, **kw) -> float:
    """Amplitude E(t) of the external field along D, 0 for t <= k*dt."""
    if t <= k * dt + 1e-12:
        return 0.0
    if kind == "sin":
        return kw.get("E0", 0.1) * math.sin(kw.get("omega", 2.0) * t)
    if kind == "gauss":
        E0, t0, s = kw.get("E0", 0.05), kw.get("t0", 2.0), kw.get("sigma", 0.5)
        return E0 * math.exp(-0.5 * ((t - t0) / s) ** 2)
    if kind == "none":
        return 0.0
    raise ValueError(kind)


def fermi(beta, w):
    x = beta * np.asarray(w, float)
    out = np.empty_like(x)
    big = np.abs(x) > 100
    out[big] = np.where(x[big] > 0, 0.0, 1.0)
    out[~big] = 1.0 / (1.0 + np.exp(x[~big]))
    return out


def fermi_exp(beta, tau, w):
    w = np.asarray(w, float)
    return np.where(w < 0, np.exp(w * tau) * fermi(beta, w), np.exp((tau - beta) * w) * fermi(beta, -w))


def hf_fock(p: Problem, rho: np.ndarray) -> np.ndarray:
    """h0 + 2J - K for the restricted density rho (molHFSolverDecomp::solve_HF, molHFSolver.cpp:81-110)."""
    V = p.Vija
    X = np.einsum("kl,kla->a", rho, V)
    J = np.einsum("ija,a->ij", V, X)
    Va = np.ascontiguousarray(V.transpose(2, 0, 1))  # V^a_ij
    K = (Va @ rho.T @ Va).sum(axis=0)                # K_ij = sum_a (V^a rho^T V^a)_ij
    return p.h0 + 2 * J - K


def uhf_fock(p: Problem, rho_up: np.ndarray, rho_dn: np.ndarray):
    """(F_up, F_dn) with F_s = h0_s + J[rho_up + rho_dn] - K[rho_s]
    (molHFSolverSpinDecomp::solve_HF, reference src/molHFSolver.cpp:203-239)."""
    V = p.Vija
    X = np.einsum("kl,kla->a", rho_up + rho_dn, V)
    J = np.einsum("ija,a->ij", V, X)
    Va = np.ascontiguousarray(V.transpose(2, 0, 1))
    out = []
    for s, rho in enumerate((rho_up, rho_dn)):
        K = (Va @ rho.T @ Va).sum(axis=0)
        out.append(p.h0_of(s) + J - K)
    return out[0], out[1]


def uhf_equilibrium(p: Problem, beta: float, iters: int = 400, tol: float = 1e-13):
    """Self-consistent unrestricted HF at inverse temperature beta: ((F_up, F_dn), (mu_up, mu_dn)),
    nao//2 electrons per spin, each mu at the mid-gap of its own spin's spectrum."""
    assert p.spin, "unrestricted equilibrium needs a spin problem"
    N = p.nao
    nocc = N // 2
    F = [p.h0.astype(complex), p.h0_dn.astype(complex)]
    mu = [0.0, 0.0]
    for _ in range(iters):
        rho = []
        for s in range(2):
            w, v = np.linalg.eigh(F[s])
            mu[s] = 0.5 * (w[nocc - 1] + w[nocc]) if 0 < nocc < N else float(w.mean())
            rho.append((v * fermi(beta, w - mu[s])) @ v.conj().T)
        Fn = uhf_fock(p, rho[0], rho[1])
        d = max(np.abs(Fn[s] - F[s]).max() for s in range(2))
        F = list(Fn)
        if d < tol:
            break
    F = [0.5 * (f + f.conj().T) for f in F]
    return (F[0].real.copy(), F[1].real.copy()), (float(mu[0]), float(mu[1]))


def hf_equilibrium(p: Problem, beta: float, iters: int = 200, tol: float = 1e-13):
    """Self-consistent restricted HF at inverse temperature beta, mu at mid-gap."""
    N = p.nao
    nocc = N // 2
    F = p.h0.astype(complex)
    mu = 0.0
    for _ in range(iters):
        w, v = np.linalg.eigh(F)
        mu = 0.5 * (w[nocc - 1] + w[nocc]) if 0 < nocc < N else float(w.mean())
        rho = (v * fermi(beta, w - mu)) @ v.conj().T
        Fn = hf_fock(p, rho)
        d = np.abs(Fn - F).max()
        F = Fn
        if d < tol:
            break
    F = 0.5 * (F + F.conj().T)
    return F.real.copy(), mu


def g0_from_h0(G: HostGF, x: np.ndarray, mu: float, H0: np.ndarray, beta: float, dt: float, k: int,
               with_matsubara: bool = True):
    """Free Green's function of a constant Hamiltonian (dyson::G0_from_h0, reference src/dyson_free.h:226-297),
    fermions (sig = -1); fills G^M (optional), G^tv(0..k,.), G^R and G^< on [0,k]^2."""
    N = G.nao
    Hmu = mu * np.eye(N) - H0
    ev, U = np.linalg.eigh(Hmu)
    evm = -ev
    Udt = (U * np.exp(1j * dt * ev)) @ U.conj().T
    Ut = [np.eye(N, dtype=complex)]
    for n in range(1, k + 1):
        Ut.append(Ut[-1] @ Udt)
    taus = beta / 2.0 * (np.asarray(x) + 1.0)
    for m, tau in enumerate(taus):
        if with_matsubara:
            G.mat[m] = -(U * fermi_exp(beta, tau, ev)) @ U.conj().T
        core = (U * fermi_exp(beta, tau, evm)) @ U.conj().T
        for n in range(k + 1):
            G.tv[n, m] = 1j * Ut[n] @ core
    val = (U * fermi(beta, evm)) @ U.conj().T
    for m in range(k + 1):
        for n in range(m + 1):
            G.retblk(m, n)[:] = -1j * Ut[m] @ Ut[n].conj().T
            G.lesblk(n, m)[:] = 1j * Ut[n] @ val @ Ut[m].conj().T


def free_history(nt: int, t_fill: int, ntau: int, x: np.ndarray, mu: float, F: np.ndarray, beta: float,
                 dt: float, scale: complex = 1.0):
    """Free (time-translation-invariant) propagation of the constant Fock matrix F on rows 0..t_fill-1,
    in packed layout: returns (les_blocks, ret_blocks, tv_rows, mat) where les/ret hold the blocks
    of the columns / rows 0..t_fill-1 (first tri(t_fill-1) blocks) and tv the rows 0..t_fill-1.
    Same closed forms as g0_from_h0: G^R(t,t') = -i U(t-t'), G^<(t',t) = i U(t'-t) f,
    G^tv(t,tau) = i U(t) e(tau), with U(n) = exp(i n dt (mu - F))."""
    N = F.shape[0]
    Hmu = mu * np.eye(N) - F
    ev, V = np.linalg.eigh(Hmu)
    n = np.arange(t_fill)
    Ud = np.einsum("ij,nj,kj->nik", V, np.exp(1j * dt * n[:, None] * ev[None, :]), V.conj())  # U(n)
    fval = (V * fermi(beta, -ev)) @ V.conj().T
    nb = t_fill * (t_fill + 1) // 2
    tt = np.repeat(n, n + 1)                     # row / column index of each packed block
    ss = np.concatenate([np.arange(t + 1) for t in n]) if t_fill > 0 else np.zeros(0, int)
    ret = -1j * Ud[tt - ss]                      # ret block (t, t') -> U(t - t')
    les = 1j * np.conj(np.transpose(Ud[tt - ss], (0, 2, 1))) @ fval   # les block (t', t): U(t'-t) f = U(t-t')^+ f
    taus = beta / 2.0 * (np.asarray(x) + 1.0)
    core = np.stack([(V * fermi_exp(beta, tau, -ev)) @ V.conj().T for tau in taus])
    tv = 1j * np.matmul(Ud[:, None], core[None])  # (t, m) -> U(t) e(tau_m), batched BLAS products
    mat = np.stack([-(V * fermi_exp(beta, tau, ev)) @ V.conj().T for tau in taus])
    return (scale * les).astype(np.complex128), (scale * ret).astype(np.complex128), \
        (scale * tv).astype(np.complex128), mat.astype(np.complex128)


def gf2_equilibrium(ctx, p: Problem, beta: float, spin: bool = False, mixing: float = 1.0, max_iter: int = 200,
                    tol: float = 1e-12):
    """Equilibrium GF2 state of problem p on the collocation grid of ctx (nedy_matsubara_gf2):
    starts from the (unrestricted) Hartree-Fock equilibrium, whose mid-gap chemical potential
    it keeps.  Returns dict(F=[Fock per spin], mu=[mu per spin], Gmat=[G^M], Smat=[Sigma^M],
    iters, diff) with host arrays; the Vija tensor of p is set on ctx."""
    import ctypes as C
    from . import api
    from ._lib import check, lib
    ns = 2 if spin else 1
    if spin:
        Fs, mus = uhf_equilibrium(p, beta)
    else:
        F, mu = hf_equilibrium(p, beta)
        Fs, mus = (F,), (mu,)
    x, _ = ctx.collocation()
    N, ntau = p.nao, ctx.ntau
    api.molGF2SolverDecomp(ctx, p.Vija)  # sets the density-fitted tensor
    Gs, Ss, h0b, Frb, Fob = [], [], [], [], []
    for s in range(ns):
        g = HostGF(-1, ntau, N, -1)
        g0_from_h0(g, x, mus[s], Fs[s], beta, 0.01, -1)
        Gs.append(api.green_func(ctx, -1, ntau, N, -1))
        Gs[-1].upload(3, 0, g.mat)
        Ss.append(api.green_func(ctx, -1, ntau, N, -1))
        h0b.append(api.DeviceBuffer.from_array(ctx, np.ascontiguousarray(p.h0_of(s) if spin else p.h0,
                                                                          dtype=np.complex128)))
        Frb.append(api.DeviceBuffer.from_array(ctx, np.ascontiguousarray(Fs[s], dtype=np.complex128)))
        Fob.append(api.DeviceBuffer(ctx, N * N * 16))
    arr = lambda objs: (C.c_void_p * ns)(*[o.h.value for o in objs])  # noqa: E731
    it, d = C.c_int(), C.c_double()
    check(lib().nedy_matsubara_gf2(ctx.h, ns, arr(Gs), arr(Ss), arr(h0b), arr(Frb), arr(Fob), float(mixing),
                                   int(max_iter), float(tol), C.byref(it), C.byref(d)))
    out = dict(mu=list(mus), iters=it.value, diff=d.value, Gmat=[], Smat=[], F=[])
    for s in range(ns):
        out["Gmat"].append(Gs[s].download(3, 0, ntau + 1))
        out["Smat"].append(Ss[s].download(3, 0, ntau + 1))
        out["F"].append(Fob[s].download((N, N)))
    return out
