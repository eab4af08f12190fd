"""Simulation drivers over the engine (host orchestration of the C ABI).

``DecompSimulation`` mirrors the reference's restricted density-fitted driver
(src/molNEsim_decomp_impl.h): ``free_gf`` + ``do_boot`` (:62-82) + ``do_tstp``
(:85-104); ``DecompSpinSimulation`` the unrestricted one
(src/molNEsim_decomp_spin_impl.h:70-122).  The equilibrium state is the
Hartree-Fock one of ``inputs.hf_equilibrium`` (the reference takes it from the
external gfmol solver), and the external drive E(t) D is added to h0 inside
h(t), gated to zero during the bootstrap window.  The unrestricted driver takes
h(t) per spin (``Problem.h0_dn``); the reference uses one hcore for both spins,
which is the case h0_dn == h0.
"""
from __future__ import annotations

import numpy as np

from . import api
from ._lib import LES, MAT, RET, TV
from .greens import HostGF
from .inputs import Problem, drive, g0_from_h0, hf_equilibrium, uhf_equilibrium


class DecompSimulation:
    def __init__(self, p: Problem, nt: int, ntau: int, beta: float, dt: float, k: int = 5,
                 corr_steps: int = 5, drive_kind: str = "none", drive_kw: dict | None = None, device: int = 0,
                 workspace_bytes: int = 0, g_window: int = 0, sigma_host: bool = False):
        """g_window > 0: G keeps only the last g_window time steps of G^R and G^< on the
        device (Sigma keeps its whole history); read each finished row with G.ret_row(t) /
        G.les_col(t) while it is in the window.  sigma_host: Sigma's two triangles in pinned
        host memory read by the kernels over the host link (runs whose history exceeds the
        device)."""
        self.p, self.nt, self.ntau, self.beta, self.dt, self.k = p, nt, ntau, beta, dt, k
        self.corr_steps = corr_steps
        self.drive_kind, self.drive_kw = drive_kind, dict(drive_kw or {})
        self.ctx = api.Context(nt, ntau, p.nao, k, beta, dt, device, workspace_bytes)
        self.x, self.w = self.ctx.collocation()
        N = p.nao
        self.G = api.green_func(self.ctx, nt, ntau, N, -1, window=g_window)
        self.Sigma = api.green_func(self.ctx, nt, ntau, N, -1, host_history=sigma_host)
        self.solver = api.molGF2SolverDecomp(self.ctx, p.Vija)
        self.dyson = api.dyson(self.ctx)
        self.hmf = api.hmf_buffer(self.ctx, N)
        self.ht = api.DeviceBuffer(self.ctx, N * N * 16)
        self.F, self.mu = hf_equilibrium(p, beta)
        self.boot_err = None

    def h_of_t(self, t: int) -> np.ndarray:
        E = drive(self.drive_kind, t * self.dt, self.k, self.dt, **self.drive_kw)
        return (self.p.h0 + E * self.p.D).astype(np.complex128)

    def set_equilibrium(self, F, Gmat):
        """Start from another equilibrium state than Hartree-Fock, e.g. the GF2 one of
        inputs.gf2_equilibrium: its Fock matrix F (mean field of the first k+1 steps) and G^M
        on the collocation grid (the free propagation of F on [0, k] stays the bootstrap guess)."""
        self.F, self._Gmat = np.asarray(F), np.asarray(Gmat)

    def initial_state(self) -> HostGF:
        g = HostGF(self.nt, self.ntau, self.p.nao, -1)
        g0_from_h0(g, self.x, self.mu, self.F, self.beta, self.dt, self.k)
        if getattr(self, "_Gmat", None) is not None:
            g.mat[:] = self._Gmat
        return g

    def free_gf(self):
        if self.G.window:
            # the initial rows 0..k only, a time step at a time
            g = HostGF(self.k, self.ntau, self.p.nao, -1)
            g0_from_h0(g, self.x, self.mu, self.F, self.beta, self.dt, self.k)
            if getattr(self, "_Gmat", None) is not None:
                g.mat[:] = self._Gmat
            for t in range(self.k + 1):
                self.G.upload(RET, t * (t + 1) // 2, g.ret_row(t))
                self.G.upload(LES, t * (t + 1) // 2, g.les_col(t))
            self.G.upload(TV, 0, g.tv)
            self.G.upload(MAT, 0, g.mat)
        else:
            self.G.from_host(self.initial_state())
        hm = np.zeros((self.nt + 1, self.p.nao, self.p.nao), np.complex128)
        hm[: self.k + 1] = self.F
        self.hmf.upload(hm)

    def do_boot(self, max_iter: int = 50, tol: float = 1e-12) -> float:
        err = None
        for _ in range(max_iter + 1):
            for t in range(self.k + 1):
                self.solver.solve(t, self.Sigma, self.G)
            err = self.dyson.dyson_start(self.G, self.Sigma, self.hmf, self.mu)
            if err < tol:
                break
        self.boot_err = err
        return err

    def do_tstp(self, t: int) -> float:
        self.ht.upload(self.h_of_t(t))
        import ctypes as C
        from ._lib import check, lib
        e = C.c_double()
        check(lib().nedy_decomp_tstp(self.ctx.h, t, self.G.h, self.Sigma.h, self.hmf.h, self.ht.h, self.mu,
                                     self.corr_steps, C.byref(e)))
        return e.value

    def do_tstp_tol(self, t: int, tol: float, max_corr: int | None = None):
        """One step with the residual exit (nedy_decomp_tstp_tol): (iterations, changes per iteration)."""
        import ctypes as C
        from ._lib import check, lib
        self.ht.upload(self.h_of_t(t))
        m = max_corr or self.corr_steps
        it = C.c_int()
        hist = (C.c_double * m)()
        check(lib().nedy_decomp_tstp_tol(self.ctx.h, t, self.G.h, self.Sigma.h, self.hmf.h, self.ht.h, self.mu, m,
                                         float(tol), C.byref(it), hist))
        return it.value, list(hist)[: it.value]

    def run(self, nt: int | None = None, boot_iter: int = 50, boot_tol: float = 1e-12):
        self.free_gf()
        self.do_boot(boot_iter, boot_tol)
        for t in range(self.k + 1, (nt if nt is not None else self.nt) + 1):
            self.do_tstp(t)


class FullSimulation:
    """Full-U restricted GF2 (reference src/molNEsim_impl.h): free_gf (:44-46), do_boot
    (:65-87, including the mixing-kernel construction set_conv_tensor at :66) and do_tstp
    (:89-124) through nedy_full_tstp.  U_ijkl = sum_Q B^Q_ij B^Q_kl and
    Uexch(j,l,n,q) = 2 U(j,n,l,q) - U(j,l,n,q) come from the problem's B^Q."""

    def __init__(self, p: Problem, nt: int, ntau: int, beta: float, dt: float, k: int = 5,
                 corr_steps: int = 5, drive_kind: str = "none", drive_kw: dict | None = None, device: int = 0):
        self.p, self.nt, self.ntau, self.beta, self.dt, self.k = p, nt, ntau, beta, dt, k
        self.corr_steps = corr_steps
        self.drive_kind, self.drive_kw = drive_kind, dict(drive_kw or {})
        self.ctx = api.Context(nt, ntau, p.nao, k, beta, dt, device)
        self.x, self.w = self.ctx.collocation()
        N = p.nao
        self.G = api.green_func(self.ctx, nt, ntau, N, -1)
        self.Sigma = api.green_func(self.ctx, nt, ntau, N, -1)
        self.solver = api.molGF2Solver(self.ctx, p.U, p.Uexch)
        self.dyson = api.dyson(self.ctx)
        self.hmf = api.hmf_buffer(self.ctx, N)
        self.ht = api.DeviceBuffer(self.ctx, N * N * 16)
        self.F, self.mu = hf_equilibrium(p, beta)
        self.boot_err = None

    def h_of_t(self, t: int) -> np.ndarray:
        E = drive(self.drive_kind, t * self.dt, self.k, self.dt, **self.drive_kw)
        return (self.p.h0 + E * self.p.D).astype(np.complex128)

    def free_gf(self):
        g = HostGF(self.nt, self.ntau, self.p.nao, -1)
        g0_from_h0(g, self.x, self.mu, self.F, self.beta, self.dt, self.k)
        self.G.from_host(g)
        hm = np.zeros((self.nt + 1, self.p.nao, self.p.nao), np.complex128)
        hm[: self.k + 1] = self.F
        self.hmf.upload(hm)

    def do_boot(self, max_iter: int = 50, tol: float = 1e-12) -> float:
        err = None
        for _ in range(max_iter + 1):
            for t in range(self.k + 1):
                self.solver.solve(t, self.Sigma, self.G)
            err = self.dyson.dyson_start(self.G, self.Sigma, self.hmf, self.mu)
            if err < tol:
                break
        self.boot_err = err
        return err

    def do_tstp(self, t: int) -> float:
        import ctypes as C
        from ._lib import check, lib
        self.ht.upload(self.h_of_t(t))
        e = C.c_double()
        check(lib().nedy_full_tstp(self.ctx.h, t, self.G.h, self.Sigma.h, self.hmf.h, self.ht.h, self.mu,
                                   self.corr_steps, C.byref(e)))
        return e.value

    def run(self, nt: int | None = None, boot_iter: int = 50, boot_tol: float = 1e-12):
        self.free_gf()
        self.do_boot(boot_iter, boot_tol)
        for t in range(self.k + 1, (nt if nt is not None else self.nt) + 1):
            self.do_tstp(t)


class DecompSpinSimulation:
    """Spin-unrestricted density-fitted GF2 (reference src/molNEsim_decomp_spin_impl.h): free_gf
    (:43-47) from the unrestricted HF equilibrium, do_boot (:63-84, the two dyson_start errors
    summed), do_tstp (:86-108) through nedy_decomp_spin_tstp, do_tstp_tol through
    nedy_decomp_spin_tstp_tol."""

    def __init__(self, p: Problem, nt: int, ntau: int, beta: float, dt: float, k: int = 5,
                 corr_steps: int = 5, drive_kind: str = "none", drive_kw: dict | None = None, device: int = 0,
                 workspace_bytes: int = 0):
        assert p.spin, "DecompSpinSimulation needs a spin problem (make_problem(..., spin=True))"
        self.p, self.nt, self.ntau, self.beta, self.dt, self.k = p, nt, ntau, beta, dt, k
        self.corr_steps = corr_steps
        self.drive_kind, self.drive_kw = drive_kind, dict(drive_kw or {})
        self.ctx = api.Context(nt, ntau, p.nao, k, beta, dt, device, workspace_bytes)
        self.x, self.w = self.ctx.collocation()
        N = p.nao
        self.G = [api.green_func(self.ctx, nt, ntau, N, -1) for _ in range(2)]
        self.Sigma = [api.green_func(self.ctx, nt, ntau, N, -1) for _ in range(2)]
        self.solver = api.molGF2SolverSpinDecomp(self.ctx, p.Vija)
        self.dyson = api.dyson(self.ctx)
        self.hmf = [api.hmf_buffer(self.ctx, N) for _ in range(2)]
        self.ht = [api.DeviceBuffer(self.ctx, N * N * 16) for _ in range(2)]
        self.F, self.mu = uhf_equilibrium(p, beta)
        self.boot_err = None

    def h_of_t(self, t: int, s: int) -> np.ndarray:
        E = drive(self.drive_kind, t * self.dt, self.k, self.dt, **self.drive_kw)
        return (self.p.h0_of(s) + E * self.p.D).astype(np.complex128)

    def initial_state(self, s: int) -> HostGF:
        g = HostGF(self.nt, self.ntau, self.p.nao, -1)
        g0_from_h0(g, self.x, self.mu[s], self.F[s], self.beta, self.dt, self.k)
        return g

    def free_gf(self):
        for s in range(2):
            self.G[s].from_host(self.initial_state(s))
            hm = np.zeros((self.nt + 1, self.p.nao, self.p.nao), np.complex128)
            hm[: self.k + 1] = self.F[s]
            self.hmf[s].upload(hm)

    def do_boot(self, max_iter: int = 50, tol: float = 1e-12) -> float:
        err = None
        for _ in range(max_iter + 1):
            for t in range(self.k + 1):
                self.solver.solve(t, self.Sigma, self.G)
            err = sum(self.dyson.dyson_start(self.G[s], self.Sigma[s], self.hmf[s], self.mu[s]) for s in range(2))
            if err < tol:
                break
        self.boot_err = err
        return err

    def _upload_h(self, t):
        for s in range(2):
            self.ht[s].upload(self.h_of_t(t, s))

    def do_tstp(self, t: int) -> float:
        import ctypes as C
        from ._lib import check, lib
        self._upload_h(t)
        e = C.c_double()
        check(lib().nedy_decomp_spin_tstp(self.ctx.h, t, self.G[0].h, self.G[1].h, self.Sigma[0].h,
                                          self.Sigma[1].h, self.hmf[0].h, self.hmf[1].h, self.ht[0].h,
                                          self.ht[1].h, self.mu[0], self.mu[1], self.corr_steps, C.byref(e)))
        return e.value

    def do_tstp_tol(self, t: int, tol: float, max_corr: int | None = None):
        """One step with the residual exit over both spins: (iterations, changes per iteration)."""
        import ctypes as C
        from ._lib import check, lib
        self._upload_h(t)
        m = max_corr or self.corr_steps
        it = C.c_int()
        hist = (C.c_double * m)()
        check(lib().nedy_decomp_spin_tstp_tol(self.ctx.h, t, self.G[0].h, self.G[1].h, self.Sigma[0].h,
                                              self.Sigma[1].h, self.hmf[0].h, self.hmf[1].h, self.ht[0].h,
                                              self.ht[1].h, self.mu[0], self.mu[1], m, float(tol), C.byref(it),
                                              hist))
        return it.value, list(hist)[: it.value]

    def run(self, nt: int | None = None, boot_iter: int = 50, boot_tol: float = 1e-12):
        self.free_gf()
        self.do_boot(boot_iter, boot_tol)
        for t in range(self.k + 1, (nt if nt is not None else self.nt) + 1):
            self.do_tstp(t)


def batch_problems(n: int, seed: int, nao_range=(8, 48), naux_per_nao: int = 4, amp_range=(0.01, 0.2),
                   freq_range=(0.5, 3.0)):
    """Seeded inputs of n independent instances: nao uniform in nao_range, naux = naux_per_nao * nao,
    each with its own h0, B^Q, dipole, and a drive E0 sin(omega t) with E0 and omega uniform in
    the given ranges.  Returns [(Problem, drive_kw)]."""
    from .inputs import make_problem
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nao = int(rng.integers(nao_range[0], nao_range[1] + 1))
        p = make_problem(nao, naux_per_nao * nao, seed=int(rng.integers(1 << 30)))
        out.append((p, {"E0": float(rng.uniform(*amp_range)), "omega": float(rng.uniform(*freq_range))}))
    return out


class BatchSimulation:
    """Many independent restricted density-fitted GF2 simulations stepped together
    (nedy_batch_tstp): each instance is a DecompSimulation with its own context; h(t) of
    every step is resident on the device (one (nt+1) x nao x nao buffer per instance)."""

    def __init__(self, problems, nt: int, ntau: int, beta: float, dt: float, k: int = 5, corr_steps: int = 5,
                 workers: int = 0, workspace_bytes: int = 1 << 30, device: int = 0, precision: int | None = None):
        from ._lib import BatchInstance
        self.nt, self.k, self.corr_steps = nt, k, corr_steps
        self.sims = [DecompSimulation(p, nt, ntau, beta, dt, k, corr_steps, "sin", kw, device, workspace_bytes)
                     for p, kw in problems]
        self.h_all = []
        for s in self.sims:
            if precision is not None:
                s.ctx.set_precision(precision)
            h = np.stack([s.h_of_t(t) for t in range(nt + 1)])
            self.h_all.append(api.DeviceBuffer.from_array(s.ctx, np.ascontiguousarray(h)))
        arr = (BatchInstance * len(self.sims))()
        for i, (s, h) in enumerate(zip(self.sims, self.h_all)):
            arr[i] = BatchInstance(s.ctx.h.value, s.G.h.value, s.Sigma.h.value, s.hmf.h.value, h.h.value, s.mu)
        self._arr = arr
        self.h = None
        self.set_workers(workers)

    def set_workers(self, workers: int):
        """(Re)create the batch with this many worker threads (<= 0: up to 16)."""
        import ctypes as C
        from ._lib import check, lib
        if getattr(self, "h", None):
            lib().nedy_batch_destroy(self.h)
        hb = C.c_void_p()
        check(lib().nedy_batch_create(self._arr, len(self.sims), int(workers), C.byref(hb)))
        self.h = hb

    def close(self):
        from ._lib import lib
        if getattr(self, "h", None):
            lib().nedy_batch_destroy(self.h)
            self.h = None
        for s in self.sims:
            s.ctx.close()

    def boot(self, max_iter: int = 50, tol: float = 1e-12):
        for s in self.sims:
            s.free_gf()
            s.do_boot(max_iter, tol)

    def do_tstp(self, t: int, tol: float = 0.0):
        """One step of every instance; returns the corrector iterations per instance."""
        import ctypes as C
        from ._lib import check, lib
        it = (C.c_int * len(self.sims))()
        check(lib().nedy_batch_tstp(self.h, int(t), int(self.corr_steps), float(tol), it))
        return list(it)
