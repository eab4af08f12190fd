#!/usr/bin/env python
"""GF2 Kadanoff-Baym time steps per second at nao=64, naux=256: plain FP64 vs
split precision + predictor at max|dG| <= 1e-8.

One "step" is one full time step T of the spin-unrestricted density-fitted GF2
simulation (DecompSpinSimulation::do_tstp, reference
src/molNEsim_decomp_spin_impl.h:86-108) through the C ABI: both spins' G rows.
Four forms run the same window from the same state (the W warm-up steps):

  split_learned_exit  the headline (value): nedy_decomp_spin_tstp_tol on a context in
                      NEDY_PREC_SPLIT_BF16X2 (or _BF16X3 with --split-mode bf16x3): the
                      self-energy contractions as BF16 piece products on tcgen05, the learned
                      predictor, and the residual exit at tol = 1e-8 (at most 5 iterations);
  split_poly_exit     the same with the polynomial predictor only;
  plain_fp64_exit     FP64 throughout with the residual exit (the exit without the precision);
  plain_fp64          nedy_decomp_spin_tstp: polynomial predictor, then CorrSteps = 5 x
                      [density matrices, unrestricted HF mean field, GF2 self-energy rows T of
                      both spins, Dyson step row T per spin], every contraction in FP64 (the
                      reference's algorithm).

The plain forms run the first --plain-steps steps of the window; every form's new rows
over those steps are compared with plain_fp64 (max |dG| per component and spin, and the
GF2 correlation energy).  e2e runs the headline form over the whole window again through
the C ABI with h(t) copied in from pinned host memory and the new G rows copied out,
inside the timed region.  --restricted runs the restricted simulation
(DecompSimulation::do_tstp, src/molNEsim_decomp_impl.h:85-104) instead.

Workload: nao=64, naux=256, independent random h0 per spin with the same B^Q, ntau=256,
beta=20, k=5, dt=0.01, steps T = t0+W ... t0+W+K-1 on a GF2 trajectory from the
unrestricted Hartree-Fock equilibrium (bootstrap, then t0-6 steps; seeded inputs, no
dataset).  The history arrays (GBs) are far larger than L2, so no explicit flush is
needed.

Multi-GPU: one independent trajectory per GPU (replicas, no collective);
value = total time steps of all ranks / max-over-ranks time.

--impl reference times the CPU restatement of the reference solver (oracle/) on the
host cores: one complete corrector iteration of the plain step at the window's first T
and the metric's ntau, measured in K parts (one per step); timesteps/s = 1 / (CorrSteps x
iteration time).  The engine arm's cpu_baseline is a bounded sample of the same
iteration (measured time per slice of each kind x slice counts, plus a Dyson step).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "GF2 timesteps/s, nao=64 naux=256: plain FP64 vs split+predictor at 1e-8"
BATCH_RESULT = [None]


def flops_sigma(T, N, A, ntau, nspin=1):
    """Algorithmic flops of one GF2 self-energy row (reference contraction order); the
    unrestricted row counts one restricted chain per spin."""
    nt1 = ntau + 1
    return nspin * ((T + 1) * (128 * N**3 * A + 44 * A * A * N * N + 36 * N**4 * A) +
                    nt1 * (36 * N**3 * A + 12 * A * A * N * N + 12 * N**4 * A))


def flops_dyson(T, N, ntau):
    """Flops of one Dyson step (history integrals, sweeps, mixing with the tau kernel)."""
    nt1 = ntau + 1
    return 8 * N**3 * (T * (T + 1) / 2 + (T + 1) ** 2 + T * T / 2 + 2 * (T + 1) * nt1 + nt1 + nt1 * nt1)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--nao", type=int, default=64)
    ap.add_argument("--naux", type=int, default=256)
    ap.add_argument("--ntau", type=int, default=256)
    ap.add_argument("--t0", type=int, default=100)
    ap.add_argument("--corr", type=int, default=5)
    ap.add_argument("--window", type=int, default=0,
                    help="keep only the last W time steps of G^R and G^< on the device (Sigma whole); "
                         "with --state synthetic the history is built on the device")
    ap.add_argument("--sigma-host", action="store_true",
                    help="Sigma's two triangles in pinned host memory (nedy_gf_create_host_history), read by "
                         "the kernels over the host link; with --window, runs whose history exceeds the device")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--tight-tol", type=float, default=1e-10,
                    help="tolerance of the predictor ablation forms (0: skip them)")
    ap.add_argument("--state", default="trajectory", choices=["trajectory", "synthetic"])
    ap.add_argument("--restricted", action="store_true",
                    help="restricted simulation instead of the spin-unrestricted one")
    ap.add_argument("--predictor", default="learned", choices=["learned", "poly"])
    ap.add_argument("--equilibrium", default="gf2", choices=["gf2", "hf"],
                    help="initial state: the GF2 equilibrium on the collocation grid (nedy_matsubara_gf2) or "
                         "the Hartree-Fock one")
    ap.add_argument("--split-mode", default="bf16x2", choices=["bf16x3", "bf16x2"],
                    help="pieces per operand of the split self-energy (bf16x2: hi*hi + hi*lo + lo*hi)")
    ap.add_argument("--split-only", action="store_true",
                    help="time the split+predictor form alone (profiling runs; no plain-form comparison)")
    ap.add_argument("--config1", action="store_true",
                    help="instead of the headline: the whole config-1 trajectory (restricted DF GF2, nao=32, "
                         "naux=128, ntau=256, beta=20, dt=0.01, nt=1000, Gaussian pulse) in FP64 on the GPU")
    ap.add_argument("--config1-nt", type=int, default=1000)
    ap.add_argument("--batch", type=int, default=64,
                    help="instances of the batched workload (0: skip it): nao uniform in [8,48], naux=4 nao")
    ap.add_argument("--batch-steps", type=int, default=3, help="timed steps of the batched workload")
    ap.add_argument("--plain-steps", type=int, default=4,
                    help="window steps of the plain FP64 forms (and of the error comparison between the forms)")
    ap.add_argument("--workspace-gb", type=float, default=0.0,
                    help="self-energy chunk workspace in GiB (0: the library default); small for profiling runs")
    ap.add_argument("--no-autotune", action="store_true",
                    help="fixed split GEMM tiles (profiling runs: the tuner's timings are meaningless under ncu)")
    ap.add_argument("--beta", type=float, default=20.0)
    ap.add_argument("--dt", type=float, default=0.01)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-seconds", type=float, default=20.0)
    return ap.parse_args()


# ------------------------------------------------------------------ distributed
class Dist:
    """One process per GPU (replicas: no data-path collective).  The process group carries
    only the barriers around the timed region and the max over ranks of the device time;
    NCCL on GPUs, gloo where no GPU is visible (the CPU tests of this logic)."""

    def __init__(self, n, backend=None, timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist
            self.backend = backend

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def replica_value(steps_per_rank: int, world: int, max_secs: float) -> float:
    """Whole-job time steps per second: every rank runs its own trajectory (weak scaling),
    timed by the slowest rank."""
    return steps_per_rank * world / max_secs


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's inputs: each replica runs an independent molecule."""
    return seed + rank


# ------------------------------------------------------------------ clocks
class Clocks:
    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU corrector iteration (oracle)
def cpu_threads():
    """Host threads for the oracle: every core, bounded by memory (each OpenMP thread holds one
    nao^4 exchange intermediate, 268 MB at nao = 64)."""
    cores = os.cpu_count() or 1
    try:
        import psutil
        mem = psutil.virtual_memory().available
        cores = max(1, min(cores, int(mem * 0.5 // (1 << 29))))
    except Exception:
        cores = min(cores, 32)
    return cores


class CpuIteration:
    """One complete corrector iteration of the plain unrestricted step at time T on the host
    cores, by the CPU restatement of the reference (oracle/): the self-energy rows of both spins
    (2 (T+1) + ntau + 1 slices, each slice both spins: reference
    src/mol2bSolver_spin_decomp_impl.h:436-466), the unrestricted mean field and one Dyson step
    per spin (src/dyson_step.h:329-382), on a free-propagation state of the workload's problem
    (rows 0..T of both spins, the metric's nao, naux and ntau).

    The iteration can run in parts (ranges of slices; the two Dyson steps in two of the parts),
    so that its complete time is measured piecewise in bounded steps."""

    def __init__(self, args, T):
        from oracle import pyoracle as po
        from nedyson_b200.greens import HostGF
        from nedyson_b200.inputs import make_problem, uhf_equilibrium, hf_equilibrium, free_history
        self.po = po
        self.cores = cpu_threads()
        po.set_threads(self.cores)
        N, A, ntau = args.nao, args.naux, args.ntau
        self.T, self.N, self.ntau, self.args = T, N, ntau, args
        self.ns = 1 if args.restricted else 2
        p = make_problem(N, A, args.seed, spin=self.ns == 2)
        if self.ns == 2:
            Fs, mus = uhf_equilibrium(p, args.beta)
        else:
            F, mu = hf_equilibrium(p, args.beta)
            Fs, mus = (F,), (mu,)
        self.mus, self.Fs, self.p = mus, Fs, p
        x, _ = po.colloc_nodes(ntau)
        self.G, self.S, self.hmf = [], [], []
        for s in range(self.ns):
            G = HostGF(T, ntau, N, -1)
            les, ret, tv, mat = free_history(T, T + 1, ntau, x, mus[s], Fs[s], args.beta, args.dt)
            G.les[:] = les
            G.ret[:] = ret
            G.tv[:] = tv
            G.mat[:] = mat
            del les, ret, tv
            S = HostGF(T, ntau, N, -1)
            S.les[:] = 0.02 * G.les
            S.ret[:] = 0.02 * G.ret
            S.tv[:] = 0.02 * G.tv
            self.G.append(G)
            self.S.append(S)
            self.hmf.append(np.repeat(Fs[s][None].astype(complex), T + 1, axis=0))
        self.df = po.DF(p.Vija)
        self.dy = po.Dyson(T, ntau, N, 5)
        nles = T + 1
        # slice jobs of the row (lesser t, retarded t, mixed tau) and their relative cost
        # (a retarded slice is two bubble and two exchange units, the others one each)
        self.njobs = 2 * nles + ntau + 1
        self.weight = np.array([1.0] * nles + [2.0] * nles + [1.0] * (ntau + 1))

    def run_jobs(self, lo, hi):
        if self.ns == 2:
            self.df.solve_spin_jobs(self.T, self.S, self.G, lo, hi)
        else:
            self.df.solve_jobs(self.T, self.S[0], self.G[0], lo, hi)

    def run_dyson(self, s):
        a = self.args
        self.dy.dyson_step(self.T, self.G[s], self.S[s], self.hmf[s], self.mus[s], a.beta, a.dt)

    def run_mean_field(self):
        rho = np.stack([g.get_dm(self.T) for g in self.G])
        if self.ns == 2:
            hu, hd = self.hmf[0][self.T].copy(), self.hmf[1][self.T].copy()
            self.df.hf_spin(hu, hd, rho)
        else:
            h = self.hmf[0][self.T].copy()
            self.df.hf(h, rho[0])

    def parts(self, n):
        """n parts of one iteration: contiguous slice ranges of equal cost; Dyson step of spin s
        in part (s + 1) n // (ns + 1); the mean field in part 0."""
        cw = np.concatenate([[0.0], np.cumsum(self.weight)])
        bounds = [int(np.searchsorted(cw, cw[-1] * i / n)) for i in range(n + 1)]
        bounds[0], bounds[-1] = 0, self.njobs
        out = []
        for i in range(n):
            dys = [s for s in range(self.ns) if (s + 1) * n // (self.ns + 1) == i] if n > 1 else list(range(self.ns))
            out.append((bounds[i], bounds[i + 1], dys, i == 0))
        return out

    def run_part(self, part):
        lo, hi, dys, mf = part
        t0 = time.perf_counter()
        if mf:
            self.run_mean_field()
        if hi > lo:
            self.run_jobs(lo, hi)
        for s in dys:
            self.run_dyson(s)
        return time.perf_counter() - t0

    def sample(self, budget_s=20.0):
        """Bounded sample of the iteration for the engine arm: the first `cores` slices of each
        kind (lesser, retarded, mixed) and one Dyson step, each timed; the iteration time is
        the measured time per slice of each kind times its slice count, plus the Dyson step
        once per spin.  Returns (iteration seconds, description)."""
        nles, ntv = self.T + 1, self.ntau + 1
        c = max(1, min(self.cores, nles, ntv))
        kinds = [("lesser", 0, nles), ("retarded", nles, nles), ("mixed", 2 * nles, ntv)]
        total, parts = 0.0, []
        for name, lo, cnt in kinds:
            t0 = time.perf_counter()
            self.run_jobs(lo, lo + c)
            dtk = time.perf_counter() - t0
            total += dtk / c * cnt
            parts.append(f"{c} {name} slices {dtk:.2f} s")
        t0 = time.perf_counter()
        self.run_dyson(0)
        dd = time.perf_counter() - t0
        total += dd * self.ns
        parts.append(f"Dyson step {dd:.2f} s (x{self.ns} spins)")
        desc = (f"oracle (C++ restatement, OpenMP over slices, OpenBLAS) on {self.cores} threads, at the bench "
                f"state's T={self.T}, ntau={self.ntau}, nao={self.N}, naux={self.args.naux}: "
                + ", ".join(parts) + f"; one iteration = measured time per slice x slice count "
                f"({2 * nles + ntv} slices per spin pair) + the Dyson steps = {total:.1f} s; one step = "
                f"{self.args.corr} iterations (the reference's CorrSteps)")
        return total, desc


def cpu_baseline_obj(value, cores, sample):
    return {"value": value, "unit": "timesteps/s", "cores": cores, "kind": "port", "sample": sample}


# DRAM bytes of all split GEMM launches per exchange unit (one slice of one spin) at nao=64,
# naux=256 with two pieces per operand: sum over the GEMM classes of dram__bytes_read.sum +
# dram__bytes_write.sum from the ncu capture of the ntau=32 case, divided by its units.
SPLIT_TRAFFIC_PER_UNIT = 3.6e8

# ------------------------------------------------------------------ peaks
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return json.load(open(path)), "measured"
        except Exception:
            pass
    # no measured file: the pool's earlier measurement (burst 1.59 PFLOP/s; sustained under the
    # power cap about 1.4 PFLOP/s)
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_gemm_peak(device: int) -> float:
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s), burst: torch.matmul float64 8192^3, best of 5."""
    import torch
    dev = torch.device(f"cuda:{device}")
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n**3 / best / 1e12


def _dev_view(ptr: int, shape, torch):
    """A complex128 torch view of engine device memory (CUDA array interface)."""
    class _A:
        __cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<c16", "data": (int(ptr), False),
                                    "version": 3}
    return torch.as_tensor(_A(), device="cuda")


def fill_synthetic_windowed(G, S, t_first, ntau, x, mu, F, beta, dt, window):
    """Free propagation of F on rows 0..t_first-1 (the closed forms of inputs.free_history:
    G^R(t,t') = -i U(t-t'), G^<(t',t) = i U(t-t')^+ f, G^tv(t,tau) = i U(t) e(tau)), written
    on the device: Sigma = 0.02 G on its full triangles and tv rows, G on its window of rows
    and its tv rows."""
    import ctypes as C
    import torch
    from nedyson_b200._lib import LES, RET, TV, MAT, check, lib
    from nedyson_b200.inputs import fermi, fermi_exp
    N = F.shape[0]
    es = N * N
    ev, V = np.linalg.eigh(mu * np.eye(N) - F)
    Vt = torch.from_numpy(V.astype(np.complex128)).cuda()
    evt = torch.from_numpy(ev).cuda()
    d = torch.arange(t_first, device="cuda", dtype=torch.float64)
    U = (Vt[None] * torch.exp(1j * dt * d[:, None] * evt[None, :])[:, None, :]) @ Vt.conj().T[None]  # U(d)
    fval = torch.from_numpy(((V * fermi(beta, -ev)) @ V.conj().T).astype(np.complex128)).cuda()
    Eret = -1j * U
    Eles = 1j * U.conj().transpose(1, 2) @ fval
    taus = beta / 2.0 * (np.asarray(x) + 1.0)
    core = torch.from_numpy(np.stack([(V * fermi_exp(beta, tau, -ev)) @ V.conj().T
                                      for tau in taus]).astype(np.complex128)).cuda()
    mat = np.stack([-(V * fermi_exp(beta, tau, ev)) @ V.conj().T for tau in taus])
    ntri = t_first * (t_first + 1) // 2
    ptr = C.c_void_p()
    views = {}
    for comp in (LES, RET, TV):
        check(lib().nedy_gf_device_pointer(S.h, comp, C.byref(ptr)))
        views[comp] = ptr.value
    if S.host_history:  # Sigma's triangles in host memory: written through the row API
        for t in range(t_first):
            o = t * (t + 1) // 2
            S.upload(RET, o, (0.02 * Eret[:t + 1].flip(0)).cpu().numpy())
            S.upload(LES, o, (0.02 * Eles[:t + 1].flip(0)).cpu().numpy())
    else:
        Sret = _dev_view(views[RET], (ntri, N, N), torch)
        Sles = _dev_view(views[LES], (ntri, N, N), torch)
        for t in range(t_first):
            o = t * (t + 1) // 2
            Sret[o:o + t + 1] = 0.02 * Eret[:t + 1].flip(0)
            Sles[o:o + t + 1] = 0.02 * Eles[:t + 1].flip(0)
    check(lib().nedy_gf_device_pointer(G.h, TV, C.byref(ptr)))
    Gtv = _dev_view(ptr.value, (t_first, ntau + 1, N, N), torch)
    Stv = _dev_view(views[TV], (t_first, ntau + 1, N, N), torch)
    for t0 in range(0, t_first, 32):
        rows = 1j * (U[t0:t0 + 32, None] @ core[None])
        Gtv[t0:t0 + rows.shape[0]] = rows
        Stv[t0:t0 + rows.shape[0]] = 0.02 * rows
    for t in range(max(0, t_first - window + 1), t_first):
        G.upload(RET, t * (t + 1) // 2, Eret[:t + 1].flip(0).cpu().numpy())
        G.upload(LES, t * (t + 1) // 2, Eles[:t + 1].flip(0).cpu().numpy())
    G.upload(MAT, 0, mat)
    torch.cuda.synchronize()


# ------------------------------------------------------------------ engine arm
def run_engine(args, dist: Dist):
    import torch
    from nedyson_b200 import api
    from nedyson_b200._lib import LES, RET, TV, MAT, PREC_FP64, PREC_SPLIT_BF16X3, PREC_SPLIT_BF16X2, check, lib
    from nedyson_b200.inputs import make_problem, hf_equilibrium, uhf_equilibrium, free_history, drive
    PREC_SPLIT = PREC_SPLIT_BF16X2 if args.split_mode == "bf16x2" else PREC_SPLIT_BF16X3

    dev = dist.local
    torch.cuda.set_device(dev)
    if args.no_autotune:
        check(lib().nedy_split_autotune(0))
    N, A, ntau, K, W = args.nao, args.naux, args.ntau, args.steps, args.warmup
    if args.window and args.state != "synthetic":
        raise SystemExit("--window builds its state on the device: use it with --state synthetic")
    spin = not args.restricted
    ns = 2 if spin else 1
    t_first = args.t0
    T_warm = list(range(t_first, t_first + W))
    T_timed = list(range(t_first + W, t_first + W + K))
    nt = t_first + W + K
    p = make_problem(N, A, rank_seed(args.seed, dist.rank), spin=spin)
    if spin:
        Fs, mus = uhf_equilibrium(p, args.beta)
    else:
        F, mu = hf_equilibrium(p, args.beta)
        Fs, mus = (F,), (mu,)
    eq_info, Gmats = None, None
    if args.equilibrium == "gf2" and args.state == "trajectory":
        from nedyson_b200.inputs import gf2_equilibrium
        te = time.time()
        ectx = api.Context(5, ntau, N, 5, args.beta, args.dt, device=dev)
        eq = gf2_equilibrium(ectx, p, args.beta, spin=spin, tol=1e-12)
        ectx.close()
        Fs, Gmats = [np.ascontiguousarray(f) for f in eq["F"]], eq["Gmat"]
        eq_info = {"kind": "GF2 equilibrium on the collocation grid (nedy_matsubara_gf2, FP64)",
                   "iterations": eq["iters"], "last_change": eq["diff"], "seconds": time.time() - te}
    ctx = api.Context(nt, ntau, N, 5, args.beta, args.dt, device=dev,
                      workspace_bytes=int(args.workspace_gb * (1 << 30)))
    x, _ = ctx.collocation()
    G = [api.green_func(ctx, nt, ntau, N, -1, window=args.window) for _ in range(ns)]
    S = [api.green_func(ctx, nt, ntau, N, -1, host_history=args.sigma_host) for _ in range(ns)]
    solver = (api.molGF2SolverSpinDecomp if spin else api.molGF2SolverDecomp)(ctx, p.Vija)
    kk = 5
    traj = args.state == "trajectory"
    # one-body Hamiltonian of every step and spin.  Trajectory state: the Gaussian pulse
    # E0 = 0.05, t0 = 2, sigma = 0.5 along D; synthetic state: 0.1 sin(2t).
    dkind, dkw = ("gauss", {"E0": 0.05, "t0": 2.0, "sigma": 0.5}) if traj else ("sin", {})

    def h_of(t, s):
        return (p.h0_of(s) + drive(dkind, t * args.dt, kk, args.dt, **dkw) * p.D).astype(np.complex128)

    hts = [[api.DeviceBuffer.from_array(ctx, h_of(t, s)) for t in range(nt + 1)] for s in range(ns)]
    hmf = []
    prep = {}

    def step_tol(t, tol, ht=None, max_corr=None):
        it = C.c_int()
        h = [(ht[s] if ht else hts[s][t]) for s in range(ns)]
        m = max_corr or args.corr
        if spin:
            check(lib().nedy_decomp_spin_tstp_tol(ctx.h, t, G[0].h, G[1].h, S[0].h, S[1].h, hmf[0].h, hmf[1].h,
                                                  h[0].h, h[1].h, mus[0], mus[1], m, tol, C.byref(it), None))
        else:
            check(lib().nedy_decomp_tstp_tol(ctx.h, t, G[0].h, S[0].h, hmf[0].h, h[0].h, mus[0], m, tol,
                                             C.byref(it), None))
        return it.value

    def step_plain(t):
        e = C.c_double()
        if spin:
            check(lib().nedy_decomp_spin_tstp(ctx.h, t, G[0].h, G[1].h, S[0].h, S[1].h, hmf[0].h, hmf[1].h,
                                              hts[0][t].h, hts[1][t].h, mus[0], mus[1], args.corr, C.byref(e)))
        else:
            check(lib().nedy_decomp_tstp(ctx.h, t, G[0].h, S[0].h, hmf[0].h, hts[0][t].h, mus[0], args.corr,
                                         C.byref(e)))
        return args.corr

    if traj:
        # GF2 trajectory from the Hartree-Fock equilibrium: free propagation on rows 0..k as
        # the bootstrap guess, dyson_start to self-consistency, then time steps up to t0-1
        # (split form with the residual exit at 1e-10).
        for s in range(ns):
            les, ret, tv, mat = free_history(nt, kk + 1, ntau, x, mus[s], Fs[s], args.beta, args.dt)
            G[s].upload(LES, 0, les)
            G[s].upload(RET, 0, ret)
            G[s].upload(TV, 0, tv)
            G[s].upload(MAT, 0, Gmats[s] if Gmats is not None else mat)
            del les, ret, tv
            hm = np.zeros((nt + 1, N, N), np.complex128)
            hm[:kk + 1] = Fs[s]
            hmf.append(api.hmf_buffer(ctx, N, hm))
        dy = api.dyson(ctx)
        tp = time.time()
        for it in range(40):
            for t in range(kk + 1):
                solver.solve(t, S if spin else S[0], G if spin else G[0])
            berr = sum(dy.dyson_start(G[s], S[s], hmf[s], mus[s]) for s in range(ns))
            if berr < 1e-12:
                break
        ctx.set_precision(PREC_SPLIT_BF16X3)  # the same state for either split mode
        # the learned predictor is trained on this trajectory's own converged rows (the steps
        # before the window; the window itself is held out)
        hist_pred = api.Predictor(ctx, 1 << 22, seed=5) if args.predictor == "learned" else None
        for t in range(kk + 1, t_first):
            step_tol(t, 1e-10)
            if hist_pred is not None and t >= 9:
                for s in range(ns):
                    hist_pred.collect(G[s], t, 64)
        ctx.synchronize()
        prep = {"equilibrium": eq_info or "Hartree-Fock", "boot_iterations": it + 1, "boot_err": berr,
                "steps": t_first - kk - 1, "seconds": time.time() - tp}
    elif args.window:
        # the free-propagation history built on the device (the host would need the whole
        # triangles): Sigma's full triangles and both tv histories through device views, G's
        # window of rows through the row API
        for s in range(ns):
            fill_synthetic_windowed(G[s], S[s], t_first, ntau, x, mus[s], Fs[s], args.beta, args.dt, args.window)
            hm = np.zeros((nt + 1, N, N), np.complex128)
            hm[:t_first] = Fs[s]
            hmf.append(api.hmf_buffer(ctx, N, hm))
        torch.cuda.synchronize(dev)
        prep = {"state": "synthetic free propagation built on the device", "window": args.window,
                "sigma_history": "pinned host memory" if args.sigma_host else "device",
                "device_memory_used_gb": (lambda fr: (fr[1] - fr[0]) / 1e9)(torch.cuda.mem_get_info(dev))}
    else:
        for s in range(ns):
            les, ret, tv, mat = free_history(nt, t_first, ntau, x, mus[s], Fs[s], args.beta, args.dt)
            G[s].upload(LES, 0, les)
            G[s].upload(RET, 0, ret)
            G[s].upload(TV, 0, tv)
            G[s].upload(MAT, 0, mat)
            S[s].upload(LES, 0, 0.02 * les)
            S[s].upload(RET, 0, 0.02 * ret)
            S[s].upload(TV, 0, 0.02 * tv)
            del les, ret, tv
            hm = np.zeros((nt + 1, N, N), np.complex128)
            hm[:t_first] = Fs[s]
            hmf.append(api.hmf_buffer(ctx, N, hm))
    # learned predictor: trained on small trajectories the engine generates (outside the timing)
    pred, pred_info = None, None
    if args.predictor == "learned" and traj:
        tt = time.time()
        nsamp = hist_pred.samples()
        loss = hist_pred.train(3000, 2048, 1e-3)
        pred = hist_pred
        pred_info = {"data": f"rows T=9..{t_first - 1} of this trajectory (both spins, every 64th element), "
                             f"the window T>={t_first} held out", "samples": nsamp, "final_loss": loss,
                     "seconds": time.time() - tt}
    elif args.predictor == "learned":
        pred, pred_info = train_predictor(ctx, args)
    sp = C.c_void_p()
    check(lib().nedy_ctx_stream(ctx.h, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device(f"cuda:{dev}"))

    def window_rows(T_list):
        """Per step T and spin: the new row of each component (les column, ret row, tv row)."""
        return [[(G[s].les_col(t), G[s].ret_row(t), G[s].tv_row(t)) for s in range(ns)] for t in T_list]

    def energies(T_list):
        d = api.dyson(ctx)
        return [[d.energy_conv(t, S[s], G[s]) for s in range(ns)] for t in T_list]

    def set_form(prec, learned):
        ctx.set_precision(prec)
        ctx.set_predictor(pred if learned else None)

    def timed(step, T_list, split, clocks_on=True):
        """Steps between CUDA events on the engine stream (one pair per step), phase times,
        launches, clocks."""
        check(lib().nedy_ctx_set_timing(ctx.h, 1))
        clocks = Clocks(dev) if (dist.rank == 0 and clocks_on) else None
        n0 = lib().nedy_launch_count()
        if split:
            check(lib().nedy_split_stats(1, None, None))
        dist.barrier()
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(T_list) + 1)]
        ev[0].record(stream)
        # NVTX range around the timed steps (lets a profiler select exactly these launches)
        torch.cuda.nvtx.range_push("timed_split" if split else "timed_plain")
        its = []
        for i, t in enumerate(T_list):
            its.append(step(t))
            ev[i + 1].record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize(dev)
        dist.barrier()
        per = [ev[i].elapsed_time(ev[i + 1]) / 1e3 for i in range(len(T_list))]
        out = {"secs": dist.max(sum(per)), "per_step_s": per, "iters": its,
               "launches": int(lib().nedy_launch_count() - n0)}
        ms4 = (C.c_double * 4)()
        check(lib().nedy_ctx_phase_times(ctx.h, ms4))
        check(lib().nedy_ctx_set_timing(ctx.h, 0))
        out["phase_ms"] = list(ms4)
        if split:
            fl, ms = C.c_double(), C.c_double()
            check(lib().nedy_split_stats(0, C.byref(fl), C.byref(ms)))
            out["split_flops"], out["split_ms"] = fl.value, ms.value
        out["clocks"] = clocks.stop() if clocks else None
        return out

    split_step = lambda t: step_tol(t, args.tol)  # noqa: E731
    exit_plain = lambda t: step_tol(t, args.tol)  # noqa: E731
    # warm-up: W steps of the headline form; their rows are the history every form starts from
    set_form(PREC_SPLIT, pred is not None)
    for t in T_warm:
        split_step(t)
    ctx.synchronize()
    Kc = min(K, args.plain_steps)  # steps compared between the forms (the plain FP64 form is slow)
    forms = {}
    # 1. headline: split precision + learned predictor + residual exit
    head = timed(split_step, T_timed, True)
    rows_head, e_head = window_rows(T_timed[:Kc]), energies(T_timed[:Kc])
    pstats = ctx.predictor_stats() if pred is not None else None
    forms["split_learned_exit"] = head
    rows, ens = {}, {}
    rows["split_learned_exit"], ens["split_learned_exit"] = rows_head, e_head
    if not args.split_only:
        # 2. split precision + polynomial predictor + residual exit
        set_form(PREC_SPLIT, False)
        forms["split_poly_exit"] = timed(split_step, T_timed, True, clocks_on=False)
        rows["split_poly_exit"], ens["split_poly_exit"] = window_rows(T_timed[:Kc]), energies(T_timed[:Kc])
        if pred is not None and args.tight_tol > 0:
            # predictor ablation at a tolerance where the prediction error decides the
            # iteration count: learned and polynomial prediction, same steps, same exit
            Tt = T_timed[:max(Kc, min(K, 10))]
            tight_step = lambda t: step_tol(t, args.tight_tol)  # noqa: E731
            for name, learned in (("split_learned_exit_tight", True), ("split_poly_exit_tight", False)):
                set_form(PREC_SPLIT, learned)
                forms[name] = timed(tight_step, Tt, True, clocks_on=False)
                forms[name]["tol"] = args.tight_tol
                if learned:
                    forms[name]["predictor_stats"] = ctx.predictor_stats()
                rows[name], ens[name] = window_rows(T_timed[:Kc]), energies(T_timed[:Kc])
        # 3. plain FP64 + residual exit (the exit alone, same arithmetic as the reference)
        set_form(PREC_FP64, False)
        forms["plain_fp64_exit"] = timed(exit_plain, T_timed[:Kc], False, clocks_on=False)
        rows["plain_fp64_exit"], ens["plain_fp64_exit"] = window_rows(T_timed[:Kc]), energies(T_timed[:Kc])
        # 4. plain FP64, CorrSteps fixed iterations: the reference's algorithm
        forms["plain_fp64"] = timed(step_plain, T_timed[:Kc], False)
        rows["plain_fp64"], ens["plain_fp64"] = window_rows(T_timed[:Kc]), energies(T_timed[:Kc])
    comps = ("les", "ret", "tv")
    spins = ("up", "down") if spin else ("restricted",)
    errs = {}
    if "plain_fp64" in rows:
        ref_rows, ref_e = rows["plain_fp64"], ens["plain_fp64"]
        for name in rows:
            if name == "plain_fp64":
                continue
            err = {}
            for si, sn in enumerate(spins):
                for ci, cn in enumerate(comps):
                    err[f"{cn}_{sn}"] = max(float(np.abs(a[si][ci] - b[si][ci]).max())
                                            for a, b in zip(ref_rows, rows[name]))
                err[f"energy_{sn}"] = max(abs(a[si] - b[si]) for a, b in zip(ref_e, ens[name]))
            err["max_abs_dG"] = max(v for k2, v in err.items() if not k2.startswith("energy"))
            errs[name] = err
    max_g = max(float(np.abs(c).max()) for r in rows_head for sr in r for c in sr)

    # end-to-end pass through the C ABI with host buffers (headline form): every step of the
    # window again, each step copying h(t) of each spin from pinned host memory in and the
    # step's new G rows (les column, ret row, tv row) back out, inside the timed region.
    set_form(PREC_SPLIT, pred is not None)
    es = N * N * 16
    h_host = torch.empty((K, ns, N, N), dtype=torch.complex128).pin_memory()
    for i, t in enumerate(T_timed):
        for s in range(ns):
            h_host[i, s].copy_(torch.from_numpy(h_of(t, s)))
    row_blocks = 2 * (nt + 1) + (ntau + 1)
    row_host = torch.empty((ns, row_blocks, N, N), dtype=torch.complex128).pin_memory()
    ht_e2e = [api.DeviceBuffer(ctx, es) for _ in range(ns)]
    h2d = d2h = 0
    dist.barrier()
    torch.cuda.synchronize(dev)
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record(stream)
    for i, t in enumerate(T_timed):
        for s in range(ns):
            check(lib().nedy_buf_upload(ht_e2e[s].h, 0, es, C.c_void_p(h_host.data_ptr() + (i * ns + s) * es)))
            h2d += es
        step_tol(t, args.tol, ht_e2e)
        for s in range(ns):
            base = row_host.data_ptr() + s * row_blocks * es
            check(lib().nedy_gf_download(G[s].h, LES, t * (t + 1) // 2, t + 1, C.c_void_p(base)))
            check(lib().nedy_gf_download(G[s].h, RET, t * (t + 1) // 2, t + 1, C.c_void_p(base + (t + 1) * es)))
            check(lib().nedy_gf_download(G[s].h, TV, t * (ntau + 1), ntau + 1,
                                         C.c_void_p(base + 2 * (t + 1) * es)))
            d2h += (2 * (t + 1) + ntau + 1) * es
    ee1.record(stream)
    torch.cuda.synchronize(dev)
    dist.barrier()
    e2e_secs = dist.max(ee0.elapsed_time(ee1) / 1e3)
    rep = C.create_string_buffer(16384)
    check(lib().nedy_split_tune_report(rep, 16384))
    tune = [x for x in rep.value.decode().split(";") if x]
    return dict(forms=forms, errs=errs, max_g=max_g, T=T_timed, Kc=Kc, e2e_secs=e2e_secs, h2d=h2d // K,
                d2h=d2h // K, prep=prep, pred_info=pred_info, pred_stats=pstats, tune=tune, mu=list(mus))


def run_batch(args, dist: Dist):
    """The batched workload: independent density-fitted GF2 instances of uneven size (nao
    uniform in [8, 48], naux = 4 nao, own h0, B^Q and dipole each, drive E0 sin(omega t) with
    E0 in [0.01, 0.2] and omega in [0.5, 3]; beta=10, ntau=128, k=5, dt=0.02), stepped
    together by nedy_batch_tstp (split-precision self-energy, residual exit at args.tol).
    After the bootstrap and a few steps, the same window runs batched (worker pool, one
    stream per instance) and one instance at a time; time on the device (events on the
    legacy stream, which every instance stream synchronises with)."""
    import torch
    from nedyson_b200._lib import PREC_SPLIT_BF16X2
    from nedyson_b200.simulation import BatchSimulation, batch_problems
    import ctypes as C
    from nedyson_b200._lib import check, lib
    n, Kb, Wb = args.batch, args.batch_steps, 2
    t_first = 6 + 2
    W_max = 24  # warm-up steps at most: the autotuner times the candidates of every instance's classes
    nt = t_first + W_max + Kb
    probs = batch_problems(n, seed=rank_seed(args.seed + 1000, dist.rank))
    tp = time.time()
    b = BatchSimulation(probs, nt, 128, 10.0, 0.02, k=5, corr_steps=5, workers=16, workspace_bytes=1 << 30,
                        device=dist.local, precision=PREC_SPLIT_BF16X2)
    b.boot(max_iter=20)
    pending = C.c_int(0)
    t = 6
    # warm up until every problem class has chosen its tile shape (a run of nt=500 steps spends
    # its first few steps there), then time steady-state steps; every rank takes the same number
    # of steps
    while t < t_first + W_max:
        b.do_tstp(t, args.tol)
        t += 1
        check(lib().nedy_split_tune_pending(C.byref(pending)))
        if t >= t_first + Wb and dist.max(float(pending.value)) == 0:
            break
    torch.cuda.synchronize()
    prep = time.time() - tp
    T_win = list(range(t, t + Kb))
    out = {}
    for mode, workers in (("batched", 16), ("one_at_a_time", 1)):
        b.set_workers(workers)
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        its = []
        for t in T_win:
            its.append(b.do_tstp(t, args.tol))
        e1.record()
        torch.cuda.synchronize()
        dist.barrier()
        secs = dist.max(e0.elapsed_time(e1) / 1e3)
        out[mode] = {"timesteps_s": Kb / secs, "instance_timesteps_s": Kb * n / secs, "ms_per_step": secs / Kb * 1e3,
                     "mean_iterations": float(np.mean(its))}
    naos = [p.nao for p, _ in probs]
    res = {"workload": f"{n} independent density-fitted GF2 instances, nao uniform in [8,48] (seeded: min {min(naos)}, "
                       f"max {max(naos)}, mean {np.mean(naos):.1f}), naux=4 nao, beta=10, ntau=128, k=5, dt=0.02, "
                       f"E0 sin(omega t) drives; steps T={T_win[0]}..{T_win[-1]} after the bootstrap; split "
                       f"self-energy (two BF16 pieces), residual exit at tol={args.tol:g}",
           "batched": out["batched"], "one_at_a_time": out["one_at_a_time"],
           "speedup_batched": out["batched"]["timesteps_s"] / out["one_at_a_time"]["timesteps_s"],
           "workers": 16, "preparation_s": prep, "warmup_steps": T_win[0] - 6,
           "tuning_classes_pending": pending.value,
           "note": "the window is short (nt=500 of the configuration needs about 0.6 TB of Green's-function history)"}
    b.close()
    return res


def run_config1(args):
    """Config 1 at its stated sizes: restricted density-fitted GF2, nao=32, naux=128, ntau=256,
    beta=20, k=5, dt=0.01, Gaussian pulse E0=0.05 t0=2 sigma=0.5 along D, FP64 throughout, from
    the GF2 equilibrium: bootstrap, then every step to nt with the reference's 5 corrector
    iterations (nedy_decomp_tstp).  Reports timesteps/s over the whole trajectory (device
    time), the energies at the end and the device memory the run held."""
    import torch
    from nedyson_b200 import api
    from nedyson_b200.inputs import make_problem, gf2_equilibrium
    from nedyson_b200.simulation import DecompSimulation
    nt, ntau, beta, dt = args.config1_nt, 256, 20.0, 0.01
    p = make_problem(32, 128, args.seed)
    t0 = time.time()
    ectx = api.Context(5, ntau, 32, 5, beta, dt)
    eq = gf2_equilibrium(ectx, p, beta)
    ectx.close()
    sim = DecompSimulation(p, nt, ntau, beta, dt, corr_steps=5, drive_kind="gauss",
                           drive_kw={"E0": 0.05, "t0": 2.0, "sigma": 0.5})
    sim.set_equilibrium(eq["F"][0], eq["Gmat"][0])
    sim.free_gf()
    berr = sim.do_boot(max_iter=40)
    prep = time.time() - t0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    marks = {}
    for t in range(6, nt + 1):
        sim.do_tstp(t)
        if t in (100, 250, 500, 750, 1000):
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            marks[t] = ev
    e1.record()
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    d = api.dyson(sim.ctx)
    e_corr = d.energy_conv(nt, sim.Sigma, sim.G)
    rho = -1j * sim.G.download(0, nt * (nt + 1) // 2 + nt, 1)[0]  # rho = i sig G^<(nt, nt), sig = -1
    free, total = torch.cuda.mem_get_info()
    line = {"workload": "config 1: restricted density-fitted GF2, nao=32 naux=128 ntau=256 beta=20 k=5 dt=0.01 "
                        f"nt={nt}, Gaussian pulse E0=0.05 t0=2 sigma=0.5, FP64, 5 corrector iterations per step, "
                        "from the GF2 equilibrium",
            "steps": nt - 5, "seconds": secs, "timesteps_s": (nt - 5) / secs,
            "seconds_at": {str(t): e0.elapsed_time(ev) / 1e3 for t, ev in marks.items()},
            "equilibrium_iterations": eq["iters"], "boot_err": berr, "preparation_s": prep,
            "E_corr_at_nt": e_corr, "device_memory_used_gb": (total - free) / 1e9,
            "electrons_at_nt": float(np.trace(rho).real)}
    print(json.dumps(line), flush=True)


def train_predictor(ctx, args):
    """Train the learned predictor on short GF2 trajectories of small molecules (nao=8,
    naux=24, Gaussian pulses of different strength and width), generated by the engine
    itself with the corrector converged; returns the predictor on ctx and a summary."""
    from nedyson_b200 import api
    from nedyson_b200.inputs import make_problem
    from nedyson_b200.simulation import DecompSimulation
    t0 = time.time()
    w, n, loss = None, 0, None
    for seed, kw in [(11, {"E0": 0.1, "t0": 0.4, "sigma": 0.15}), (12, {"E0": 0.05, "t0": 0.3, "sigma": 0.1}),
                     (14, {"E0": 0.08, "t0": 0.35, "sigma": 0.08})]:
        sm = DecompSimulation(make_problem(8, 24, seed), 60, 32, 10.0, args.dt, drive_kind="gauss", drive_kw=kw,
                              device=ctx.device)
        sm.free_gf()
        sm.do_boot()
        P = api.Predictor(sm.ctx, 1 << 21, seed=5)
        if w is not None:
            P.set_params(w)
        for t in range(6, sm.nt + 1):
            sm.do_tstp_tol(t, 1e-13, 8)
            if t >= 9:
                P.collect(sm.G, t, 1)
        n += P.samples()
        loss = P.train(1500, 1024, 1e-3)
        w = P.params()
        P.close()
        sm.ctx.close()
    pred = api.Predictor(ctx, 1 << 10, seed=5)
    pred.set_params(w)
    return pred, {"trajectories": 3, "samples": n, "final_loss": loss, "seconds": time.time() - t0}


def main():
    args = parse()
    dist = Dist(args.gpus)
    K, W = args.steps, args.warmup
    kind = ("restricted density-fitted GF2 time step" if args.restricted else
            "spin-unrestricted density-fitted GF2 time step (both spins, independent h0 per spin, same B^Q)")
    cfg = {"workload": f"{kind}, nao={args.nao} naux={args.naux} ntau={args.ntau} "
                       f"beta={args.beta} k=5 dt={args.dt}, steps T={args.t0 + W}..{args.t0 + W + K - 1} on a "
                       f"pre-evolved {args.state} state",
           "nao": args.nao, "naux": args.naux, "ntau": args.ntau, "nspin": 1 if args.restricted else 2,
           "t_window": [args.t0 + W, args.t0 + W + K - 1], "corr_steps": args.corr,
           "l2": "inputs (G, Sigma histories, GBs) larger than L2; no flush needed",
           "parallelism": f"replicas x{dist.world}"}
    if args.window:
        cfg["g_window"] = args.window
    if args.sigma_host:
        cfg["sigma_history"] = "pinned host memory, read by the kernels over the host link"
    T_ref = args.t0 + W  # the first step of the window
    if args.impl == "reference":
        if dist.rank != 0:
            dist.close()
            return
        # One complete corrector iteration of the plain step at the window's first T, measured
        # in K parts (one part per step; the W warm-up steps run parts untimed first).  A time
        # step is CorrSteps such iterations, so timesteps/s = 1 / (CorrSteps x iteration time).
        it = CpuIteration(args, T_ref)
        parts = it.parts(K)
        for i in range(W):
            it.run_part(parts[i % K])
        secs = [it.run_part(pt) for pt in parts]
        t_iter = float(sum(secs))
        value = 1.0 / (args.corr * t_iter)
        sample = (f"oracle (C++ restatement of the reference, OpenMP over slices, OpenBLAS) on {it.cores} threads: "
                  f"one complete corrector iteration of the plain {'unrestricted' if it.ns == 2 else 'restricted'} "
                  f"step at T={T_ref}, ntau={args.ntau}, nao={args.nao}, naux={args.naux} (self-energy rows of "
                  f"{'both spins' if it.ns == 2 else 'the row'}: {it.njobs} slices, mean field, {it.ns} Dyson "
                  f"step{'s' if it.ns == 2 else ''}) measured in {K} parts, {t_iter:.1f} s; one time step = "
                  f"{args.corr} iterations (CorrSteps); each bench step is one part")
        cfg["precision"] = "fp64 (the reference's arithmetic)"
        cfg["predictor"] = f"polynomial extrapolation (k=5), {args.corr} corrector iterations"
        line = {"metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": 0, "steps": K, "warmup": W,
                "ms_per_step": float(np.mean(secs)) * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "complex128", "data": "synthetic (seeded)", "config": cfg,
                "impl": "reference", "full_step_ms": args.corr * t_iter * 1e3,
                "iteration_parts_s": secs,
                "cpu_baseline": cpu_baseline_obj(value, it.cores, sample),
                "e2e": {"value": value, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        dist.close()
        return

    if args.config1:
        if dist.rank == 0:
            run_config1(args)
        dist.close()
        return
    fp64 = fp64_gemm_peak(dist.local) if dist.rank == 0 else None
    r = run_engine(args, dist)
    import gc
    gc.collect()  # release the headline state before the batched workload
    if args.batch > 0 and not args.split_only:
        BATCH_RESULT[0] = run_batch(args, dist)
    fm = r["forms"]
    head = fm["split_learned_exit"]
    value = replica_value(K, dist.world, head["secs"])
    peaks, src = measured_peaks()
    cfg["precision"] = ({"bf16x2": "split self-energy, two BF16 pieces per operand, products hi*hi + hi*lo + lo*hi",
                         "bf16x3": "split self-energy, three BF16 pieces per operand, six products"}[args.split_mode] +
                        " (tcgen05, FP32 accumulation), FP64 Dyson/HF/density/residual")
    cfg["predictor"] = ("learned MLP correction of the k=5 extrapolation (polynomial fallback)" if args.predictor == "learned"
                        else "polynomial extrapolation (k=5)") + f" + residual exit at tol={args.tol:g} (at most {args.corr} iterations)"
    eqname = "GF2" if args.equilibrium == "gf2" else "HF"
    cfg["state"] = (f"GF2 trajectory from the {'restricted' if args.restricted else 'unrestricted'} {eqname} equilibrium "
                    "(Gaussian pulse E0=0.05 t0=2 sigma=0.5)"
                    if args.state == "trajectory" else "synthetic free-propagation history, 0.1 sin(2t) drive")
    cfg["tol"] = args.tol
    cfg["warmup"] = f"{W} steps of the headline form (T={args.t0}..{args.t0 + W - 1}); every form starts from them"
    line = {"metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": dist.world, "steps": K, "warmup": W,
            "ms_per_step": head["secs"] / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128 state; self-energy contractions in BF16 pieces with FP32 accumulation",
            "data": ("synthetic (seeded random h0, B^Q, dipole); state: " + cfg["state"]), "config": cfg}
    if dist.rank == 0:
        # dominant kernel of the headline form: the split GEMM (BF16 piece products on tcgen05);
        # achieved = algorithmic BF16 pipe FLOPs / its summed device time (CUDA events per launch)
        bf16_peak = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
        ach = head["split_flops"] / (head["split_ms"] / 1e3) / 1e12 if head.get("split_ms") else None
        peak_key = "bf16_tflops_sustained" if peaks.get("bf16_tflops_sustained") else "bf16_tflops"
        nsp = 1 if args.restricted else 2
        # DRAM traffic of the split GEMMs per step: bytes per exchange unit (one slice of one
        # spin; dram__bytes_read.sum + dram__bytes_write.sum of every split GEMM class, ncu
        # capture of the nao=64, naux=256, ntau=32 case with two pieces per operand) times the
        # units of the step (les, tv and ret slices times the iterations)
        units = sum(nsp * (2 * (t + 1) + args.ntau + 1) * it for t, it in zip(r["T"], head["iters"])) / K
        per_unit = SPLIT_TRAFFIC_PER_UNIT if (args.nao, args.naux, args.split_mode) == (64, 256, "bf16x2") else None
        line["roofline"] = {"bound": "tensor", "kernel": "split GEMM kernels: split_gemm_kernel, split_gemm_persist_kernel, "
                            "split_gemm_pair_kernel, split_gemm_persist_pair_kernel (BF16 piece products, "
                            "tcgen05, TMEM; every launch of the step)",
                            "achieved": ach, "peak": bf16_peak, "unit": "TFLOP/s",
                            "frac": (ach / bf16_peak) if ach else None,
                            "traffic": per_unit * units if per_unit else None,
                            "traffic_unit": "bytes per step (DRAM, all split GEMM launches of one step)",
                            "exchange_units_per_step": units,
                            "peak_source": f"{src}: {peak_key} (kernel timed inside a long step)",
                            "algorithmic_flops_per_step": head["split_flops"] / K,
                            "kernel_ms_per_step": head["split_ms"] / K}
        Kc = r["Kc"]

        def form_obj(f, name):
            n = len(f["per_step_s"])
            o = {"timesteps_s": n / f["secs"], "ms_per_step": f["secs"] / n * 1e3, "steps": n,
                 "iterations_per_step": f["iters"], "mean_iterations": float(np.mean(f["iters"])),
                 "phase_ms": dict(zip(["predictor", "mean_field", "self_energy", "dyson"], f["phase_ms"])),
                 "gpu_launches": f["launches"],
                 # the first Kc steps: the window every form ran
                 "timesteps_s_first_steps": Kc / sum(f["per_step_s"][:Kc])}
            if name in r["errs"]:
                o["error_vs_plain_fp64"] = r["errs"][name]
            for key in ("tol", "predictor_stats"):
                if key in f:
                    o[key] = f[key]
            return o

        forms = {name: form_obj(f, name) for name, f in fm.items()}
        if "plain_fp64" in fm:
            pl = fm["plain_fp64"]
            sig_flops = sum(flops_sigma(t, args.nao, args.naux, args.ntau, nsp) for t in r["T"][:Kc]) * args.corr
            forms["plain_fp64"]["self_energy_fp64_tflops"] = sig_flops / (pl["phase_ms"][2] / 1e3) / 1e12
            forms["plain_fp64"]["fp64_peak_tflops"] = fp64
            base = forms["plain_fp64"]["timesteps_s_first_steps"]
            for name in forms:
                forms[name]["speedup_vs_plain_fp64"] = forms[name]["timesteps_s_first_steps"] / base
            if "plain_fp64_exit" in forms:
                bx = forms["plain_fp64_exit"]["timesteps_s_first_steps"]
                for name in forms:
                    forms[name]["speedup_vs_plain_fp64_exit"] = forms[name]["timesteps_s_first_steps"] / bx
        line["forms"] = forms
        line["forms_note"] = (f"every form runs the window from the same state (the {W} warm-up steps); the "
                              f"plain FP64 forms and the error comparison cover the first {Kc} steps; "
                              "speedups compare timesteps/s over those common steps; errors are max |G_form - "
                              "G_plain_fp64| over the new rows of those steps (per component and spin) and "
                              "|E_corr difference| per spin")
        line["state_preparation"] = r["prep"]
        line["predictor_training"] = r["pred_info"]
        line["predictor_stats"] = r["pred_stats"]
        line["split_tile_autotune"] = r["tune"]
        line["max_abs_G"] = r["max_g"]
        line["mu"] = r["mu"]
        line["clocks"] = head["clocks"]
        if "plain_fp64" in fm:
            line["clocks_plain"] = fm["plain_fp64"]["clocks"]
        line["gpu_launches"] = head["launches"]
        line["e2e"] = {"value": replica_value(K, dist.world, r["e2e_secs"]), "unit": "timesteps/s",
                       "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                       "what": "the headline form over the whole window again through the C ABI, each step copying "
                               "h(t) of each spin in from pinned host memory and its new G rows out"}
        if args.batch > 0 and not args.split_only:
            line["batched_workload"] = BATCH_RESULT[0]
        if dist.world == 1 and not args.no_cpu_baseline:
            it = CpuIteration(args, T_ref)
            t_iter, desc = it.sample()
            line["cpu_baseline"] = cpu_baseline_obj(1.0 / (args.corr * t_iter), it.cores, desc)
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
