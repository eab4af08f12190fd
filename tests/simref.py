"""Oracle-side simulation driver used by the parity tests (test infrastructure).

Same initial state and the same do_boot / do_tstp sequence as
``nedyson_b200.simulation.DecompSimulation`` (reference
src/molNEsim_decomp_impl.h:62-104) and ``DecompSpinSimulation`` (reference
src/molNEsim_decomp_spin_impl.h:63-108), on the CPU oracle.
"""
import numpy as np

from oracle import pyoracle as po
from nedyson_b200.greens import HostGF
from nedyson_b200.inputs import Problem, drive, g0_from_h0, hf_equilibrium, uhf_equilibrium


class OracleDecompSim:
    def __init__(self, p: Problem, nt, ntau, beta, dt, k=5, corr_steps=5, drive_kind="none", drive_kw=None):
        self.p, self.nt, self.ntau, self.beta, self.dt, self.k = p, nt, ntau, beta, dt, k
        self.corr_steps = corr_steps
        self.drive_kind, self.drive_kw = drive_kind, dict(drive_kw or {})
        self.dy = po.Dyson(nt, ntau, p.nao, k)
        self.df = po.DF(p.Vija)
        self.x, _ = po.colloc_nodes(ntau)
        self.F, self.mu = hf_equilibrium(p, beta)
        self.G = HostGF(nt, ntau, p.nao, -1)
        self.S = HostGF(nt, ntau, p.nao, -1)
        self.hmf = np.zeros((nt + 1, p.nao, p.nao), np.complex128)

    def h_of_t(self, t):
        E = drive(self.drive_kind, t * self.dt, self.k, self.dt, **self.drive_kw)
        return (self.p.h0 + E * self.p.D).astype(np.complex128)

    def set_equilibrium(self, F, Gmat):
        """Start from another equilibrium state (e.g. the GF2 one): Fock matrix F, G^M on the grid."""
        self.F, self._Gmat = np.asarray(F), np.asarray(Gmat)

    def free_gf(self):
        g0_from_h0(self.G, self.x, self.mu, self.F, self.beta, self.dt, self.k)
        if getattr(self, "_Gmat", None) is not None:
            self.G.mat[:] = self._Gmat
        self.hmf[: self.k + 1] = self.F

    def do_boot(self, max_iter=50, tol=1e-12):
        err = None
        for _ in range(max_iter + 1):
            for t in range(self.k + 1):
                self.df.solve(t, self.S, self.G)
            err = self.dy.dyson_start(self.G, self.S, self.hmf, self.mu, self.beta, self.dt)
            if err < tol:
                break
        return err

    def do_tstp(self, t):
        self.dy.extrapolate(t, self.G)
        e = None
        for _ in range(self.corr_steps):
            rho = self.G.get_dm(t)
            self.hmf[t] = self.h_of_t(t)
            self.df.hf(self.hmf[t], rho)
            self.df.solve(t, self.S, self.G)
            e, _ = self.dy.dyson_step(t, self.G, self.S, self.hmf, self.mu, self.beta, self.dt)
        return e


class OracleFullSim(OracleDecompSim):
    """Full-U driver (reference src/molNEsim_impl.h:65-124) on the oracle: the same sequence
    as OracleDecompSim with molGF2Solver / molHFSolver in place of the density-fitted ones."""

    def __init__(self, p: Problem, nt, ntau, beta, dt, k=5, corr_steps=5, drive_kind="none", drive_kw=None):
        super().__init__(p, nt, ntau, beta, dt, k, corr_steps, drive_kind, drive_kw)
        self.df = _FullAsDF(po.Full(p.U, p.Uexch))


class _FullAsDF:
    """po.Full under the method names the restricted driver calls."""

    def __init__(self, full):
        self.full = full

    def solve(self, t, S, G):
        self.full.solve(t, S, G)

    def hf(self, hmf_t, rho):
        self.full.hf(hmf_t, rho)


class OracleDecompSpinSim:
    def __init__(self, p: Problem, nt, ntau, beta, dt, k=5, corr_steps=5, drive_kind="none", drive_kw=None):
        self.p, self.nt, self.ntau, self.beta, self.dt, self.k = p, nt, ntau, beta, dt, k
        self.corr_steps = corr_steps
        self.drive_kind, self.drive_kw = drive_kind, dict(drive_kw or {})
        self.dy = po.Dyson(nt, ntau, p.nao, k)
        self.df = po.DF(p.Vija)
        self.x, _ = po.colloc_nodes(ntau)
        self.F, self.mu = uhf_equilibrium(p, beta)
        self.G = [HostGF(nt, ntau, p.nao, -1) for _ in range(2)]
        self.S = [HostGF(nt, ntau, p.nao, -1) for _ in range(2)]
        self.hmf = np.zeros((2, nt + 1, p.nao, p.nao), np.complex128)

    def h_of_t(self, t, s):
        E = drive(self.drive_kind, t * self.dt, self.k, self.dt, **self.drive_kw)
        return (self.p.h0_of(s) + E * self.p.D).astype(np.complex128)

    def free_gf(self):
        for s in range(2):
            g0_from_h0(self.G[s], self.x, self.mu[s], self.F[s], self.beta, self.dt, self.k)
            self.hmf[s, : self.k + 1] = self.F[s]

    def do_boot(self, max_iter=50, tol=1e-12):
        err = None
        for _ in range(max_iter + 1):
            for t in range(self.k + 1):
                self.df.solve_spin(t, self.S, self.G)
            err = sum(self.dy.dyson_start(self.G[s], self.S[s], self.hmf[s], self.mu[s], self.beta, self.dt)
                      for s in range(2))
            if err < tol:
                break
        return err

    def do_tstp(self, t):
        for s in range(2):
            self.dy.extrapolate(t, self.G[s])
        for _ in range(self.corr_steps):
            rho2 = np.stack([self.G[s].get_dm(t) for s in range(2)])
            hu, hd = self.h_of_t(t, 0), self.h_of_t(t, 1)
            self.df.hf_spin(hu, hd, rho2)
            self.hmf[0, t], self.hmf[1, t] = hu, hd
            self.df.solve_spin(t, self.S, self.G)
            for s in range(2):
                self.dy.dyson_step(t, self.G[s], self.S[s], self.hmf[s], self.mu[s], self.beta, self.dt)
