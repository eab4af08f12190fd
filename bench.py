#!/usr/bin/env python
"""GF2 Kadanoff-Baym time steps per second at nao=64, naux=256: plain FP64 vs
split precision + predictor at max|dG| <= 1e-8.

One "step" is one full time step T of the spin-unrestricted density-fitted GF2
simulation (DecompSpinSimulation::do_tstp, reference
src/molNEsim_decomp_spin_impl.h:86-108) through the C ABI: both spins' G rows.
Two forms run the same window from the same state:

  plain FP64       nedy_decomp_spin_tstp: polynomial predictor, then CorrSteps = 5 x
                   [density matrices, unrestricted HF mean field, GF2 self-energy rows T
                   of both spins, Dyson step row T per spin], every contraction in FP64
                   (the reference's algorithm);
  split+predictor  nedy_decomp_spin_tstp_tol on a context in NEDY_PREC_SPLIT_BF16X2 (or
                   _BF16X3 with --split-mode bf16x3): the self-energy contractions as
                   BF16 piece products on tcgen05, the
                   predictor, and the residual exit at tol = 1e-8 (at most 5 iterations).

value is the split+predictor form (the headline); the plain form, the iterations per
step and max|dG| between the two forms over the window (per component and spin, and
the GF2 correlation energy) are in the same line.  --restricted runs the restricted
simulation (DecompSimulation::do_tstp, src/molNEsim_decomp_impl.h:85-104) instead.

Workload: nao=64, naux=256, independent random h0 per spin with the same B^Q, ntau=256,
beta=20, k=5, dt=0.01, steps T = t0+W ... t0+W+K-1 on a GF2 trajectory from the
unrestricted Hartree-Fock equilibrium (bootstrap, then t0-6 steps; seeded inputs, no
dataset).  The history arrays (GBs) are far larger than L2, so no explicit flush is
needed.

Multi-GPU: one independent trajectory per GPU (replicas, no collective);
value = total time steps of all ranks / max-over-ranks time.

--impl reference times the CPU restatement of the reference solver (oracle/)
on the host cores on a bounded sample and reports the same metric.
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
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--state", default="trajectory", choices=["trajectory", "synthetic"])
    ap.add_argument("--restricted", action="store_true",
                    help="restricted simulation instead of the spin-unrestricted one")
    ap.add_argument("--predictor", default="learned", choices=["learned", "poly"])
    ap.add_argument("--split-mode", default="bf16x2", choices=["bf16x3", "bf16x2"],
                    help="pieces per operand of the split self-energy (bf16x2: hi*hi + hi*lo + lo*hi)")
    ap.add_argument("--split-only", action="store_true",
                    help="time the split+predictor form alone (profiling runs; no plain-form comparison)")
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


# ------------------------------------------------------------------ CPU sample (oracle)
def cpu_sample(args, target_seconds=20.0):
    """Time the CPU restatement of the reference on a bounded sample and scale to one step at T.

    Sample: one GF2 self-energy row at (nao, naux) with small T_s / ntau_s (enough slices for
    every core), and one Dyson step at T_d = 24, ntau_d = 16; each is scaled to the bench
    step by the flop models above (time per flop assumed constant)."""
    from oracle import pyoracle as po
    from nedyson_b200.greens import HostGF
    from nedyson_b200.inputs import make_problem, hf_equilibrium, free_history
    # every OpenMP thread holds one nao^4 exchange intermediate (268 MB at nao = 64): cap the threads
    cores = min(os.cpu_count() or 1, 32)
    po.set_threads(cores)
    N, A = args.nao, args.naux
    ns = 1 if args.restricted else 2
    p = make_problem(N, A, args.seed, spin=ns == 2)
    rng = np.random.default_rng(1)
    ntau_s = 8
    T_s = max(2, (cores - ntau_s - 1 + 1) // 2)
    Gs, Ss = [], []
    for _ in range(ns):
        G = HostGF(T_s, ntau_s, N, -1)
        for a in (G.les, G.ret, G.tv):
            a[:] = 0.05 * (rng.uniform(-1, 1, a.shape) + 1j * rng.uniform(-1, 1, a.shape))
        Gs.append(G)
        Ss.append(HostGF(T_s, ntau_s, N, -1))
    df = po.DF(p.Vija)
    t0 = time.perf_counter()
    if ns == 2:
        df.solve_spin(T_s, Ss, Gs)
    else:
        df.solve(T_s, Ss[0], Gs[0])
    ts = time.perf_counter() - t0
    rate_s = flops_sigma(T_s, N, A, ntau_s, ns) / ts
    # Dyson sample
    T_d, ntau_d = 24, 16
    F, mu = hf_equilibrium(make_problem(N, A, args.seed), args.beta)
    x, _ = po.colloc_nodes(ntau_d)
    Gd = HostGF(T_d, ntau_d, N, -1)
    les, ret, tv, mat = free_history(T_d, T_d + 1, ntau_d, x, mu, F, args.beta, args.dt)
    Gd.les[:] = les
    Gd.ret[:] = ret
    Gd.tv[:] = tv
    Gd.mat[:] = mat
    Sd = HostGF(T_d, ntau_d, N, -1)
    Sd.les[:] = 0.02 * les
    Sd.ret[:] = 0.02 * ret
    Sd.tv[:] = 0.02 * tv
    hmf = np.repeat(F[None].astype(complex), T_d + 1, axis=0)
    dy = po.Dyson(T_d, ntau_d, N, 5)
    dy.mixing(Sd.tv[0], Gd.mat, args.beta, -1.0)  # builds the tau kernel outside the timing
    t0 = time.perf_counter()
    dy.dyson_step(T_d, Gd, Sd, hmf, mu, args.beta, args.dt)
    td = time.perf_counter() - t0
    rate_d = flops_dyson(T_d, N, ntau_d) / td
    return dict(cores=cores, T_s=T_s, ntau_s=ntau_s, sigma_s=ts, rate_sigma=rate_s, T_d=T_d, ntau_d=ntau_d,
                dyson_s=td, rate_dyson=rate_d, nspin=ns)


def cpu_step_seconds(smp, T, args):
    """One step: CorrSteps x (self-energy rows of all spins + one Dyson step per spin)."""
    ns = smp["nspin"]
    return args.corr * (flops_sigma(T, args.nao, args.naux, args.ntau, ns) / smp["rate_sigma"] +
                        ns * flops_dyson(T, args.nao, args.ntau) / smp["rate_dyson"])


def cpu_baseline_obj(smp, value, args):
    return {"value": value, "unit": "timesteps/s", "cores": smp["cores"], "kind": "port",
            "sample": (f"oracle (C++ restatement, OpenMP over slices, OpenBLAS) timed on one "
                       f"{'unrestricted (both spins)' if smp['nspin'] == 2 else 'restricted'} GF2 self-energy row "
                       f"at nao={args.nao}, naux={args.naux}, T={smp['T_s']}, ntau={smp['ntau_s']} "
                       f"({smp['sigma_s']:.2f} s, {smp['rate_sigma'] / 1e9:.1f} GFLOP/s) and one Dyson step at "
                       f"T={smp['T_d']}, ntau={smp['ntau_d']} ({smp['dyson_s']:.2f} s, "
                       f"{smp['rate_dyson'] / 1e9:.1f} GFLOP/s), scaled by the flop model to one "
                       f"{args.corr}-iteration step ({smp['nspin']} Dyson steps per iteration) at T={args.t0 + args.warmup}, "
                       f"ntau={args.ntau}")}


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
    spin = not args.restricted
    ns = 2 if spin else 1
    t_first = args.t0
    nt = t_first + W + K
    p = make_problem(N, A, rank_seed(args.seed, dist.rank), spin=spin)
    if spin:
        Fs, mus = uhf_equilibrium(p, args.beta)
    else:
        F, mu = hf_equilibrium(p, args.beta)
        Fs, mus = (F,), (mu,)
    ctx = api.Context(nt, ntau, N, 5, args.beta, args.dt, device=dev,
                      workspace_bytes=int(args.workspace_gb * (1 << 30)))
    x, _ = ctx.collocation()
    G = [api.green_func(ctx, nt, ntau, N, -1) for _ in range(ns)]
    S = [api.green_func(ctx, nt, ntau, N, -1) for _ in range(ns)]
    solver = (api.molGF2SolverSpinDecomp if spin else api.molGF2SolverDecomp)(ctx, p.Vija)
    kk = 5
    traj = args.state == "trajectory"
    # one-body Hamiltonian of every step and spin, resident on the device.  Trajectory state:
    # the Gaussian pulse E0 = 0.05, t0 = 2, sigma = 0.5 along D; synthetic state: 0.1 sin(2t).
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

    if traj:
        # GF2 trajectory from the Hartree-Fock equilibrium: free propagation on rows 0..k as
        # the bootstrap guess, dyson_start to self-consistency, then time steps up to t0-1
        # (split form with the residual exit at 1e-10).
        for s in range(ns):
            les, ret, tv, mat = free_history(nt, kk + 1, ntau, x, mus[s], Fs[s], args.beta, args.dt)
            G[s].upload(LES, 0, les)
            G[s].upload(RET, 0, ret)
            G[s].upload(TV, 0, tv)
            G[s].upload(MAT, 0, mat)
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
        for t in range(kk + 1, t_first):
            step_tol(t, 1e-10)
        ctx.synchronize()
        prep = {"boot_iterations": it + 1, "boot_err": berr, "steps": t_first - kk - 1,
                "seconds": time.time() - tp}
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
    if args.predictor == "learned":
        pred, pred_info = train_predictor(ctx, args)
    # pinned host buffers for the end-to-end pass: h(t) of each spin in, new G rows out
    row_blocks = 2 * (nt + 1) + (ntau + 1)
    h_host = torch.empty((ns, N, N), dtype=torch.complex128).pin_memory()
    row_host = torch.empty((ns, row_blocks, N, N), dtype=torch.complex128).pin_memory()
    ht_e2e = [api.DeviceBuffer(ctx, N * N * 16) for _ in range(ns)]
    sp = C.c_void_p()
    check(lib().nedy_ctx_stream(ctx.h, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device(f"cuda:{dev}"))
    iters = []

    def step_plain(t):
        e = C.c_double()
        if spin:
            check(lib().nedy_decomp_spin_tstp(ctx.h, t, G[0].h, G[1].h, S[0].h, S[1].h, hmf[0].h, hmf[1].h,
                                              hts[0][t].h, hts[1][t].h, mus[0], mus[1], args.corr, C.byref(e)))
        else:
            check(lib().nedy_decomp_tstp(ctx.h, t, G[0].h, S[0].h, hmf[0].h, hts[0][t].h, mus[0], args.corr,
                                         C.byref(e)))

    def step_split(t, ht=None):
        iters.append(step_tol(t, args.tol, ht))

    def window_rows(T_list):
        """Per step T and spin: the new row of each component (les column, ret row, tv row)."""
        return [[(G[s].les_col(t), G[s].ret_row(t), G[s].tv_row(t)) for s in range(ns)] for t in T_list]

    def energies(T_list):
        dy = api.dyson(ctx)
        return [[dy.energy_conv(t, S[s], G[s]) for s in range(ns)] for t in T_list]

    def timed(step, T_list, split):
        """K steps between CUDA events on the engine stream, phase times, launches, clocks."""
        check(lib().nedy_ctx_set_timing(ctx.h, 1))
        clocks = Clocks(dev) if dist.rank == 0 else None
        n0 = lib().nedy_launch_count()
        if split:
            check(lib().nedy_split_stats(1, None, None))
        dist.barrier()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # NVTX range around the timed steps (lets a profiler select exactly these launches)
        torch.cuda.nvtx.range_push("timed_split" if split else "timed_plain")
        for t in T_list:
            step(t)
        torch.cuda.nvtx.range_pop()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        dist.barrier()
        secs = e0.elapsed_time(e1) / 1e3
        out = {"secs": dist.max(secs), "launches": int(lib().nedy_launch_count() - n0)}
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

    T_timed = list(range(t_first + W, t_first + W + K))
    # shared warm-up: W plain steps define the starting state of both forms
    ctx.set_precision(PREC_SPLIT if args.split_only else PREC_FP64)
    for t in range(t_first, t_first + W):
        (step_split if args.split_only else step_plain)(t)
    ctx.synchronize()
    plain, rows_plain, e_plain = None, None, None
    if not args.split_only:
        plain = timed(step_plain, T_timed, False)
        rows_plain = window_rows(T_timed)
        e_plain = energies(T_timed)
    # split+predictor: warm-up on the window rows (recomputed below from the same history)
    ctx.set_precision(PREC_SPLIT)
    if pred is not None:
        ctx.set_predictor(pred)
    for t in T_timed[:W]:
        step_split(t)
    ctx.synchronize()
    iters.clear()
    split = timed(step_split, T_timed, True)
    split_iters = list(iters)
    rows_split = window_rows(T_timed)
    e_split = energies(T_timed)
    comps = ("les", "ret", "tv")
    spins = ("up", "down") if spin else ("restricted",)
    err = None
    if rows_plain:
        err = {}
        for si, sn in enumerate(spins):
            for ci, cn in enumerate(comps):
                err[f"{cn}_{sn}"] = max(float(np.abs(a[si][ci] - b[si][ci]).max())
                                        for a, b in zip(rows_plain, rows_split))
            err[f"energy_{sn}"] = max(abs(a[si] - b[si]) for a, b in zip(e_plain, e_split))
    max_dg = max(v for k, v in err.items() if not k.startswith("energy")) if err else None
    max_g = max(float(np.abs(c).max()) for r in rows_split for sr in r for c in sr)

    # end-to-end pass through the C ABI with host buffers (split form): re-run the last timed
    # step T_e (rows are recomputed in place), copying h(T_e) of each spin from pinned host
    # memory in and the new G rows (les column, ret row, tv row) back out, all inside the
    # timed region.
    T_e = T_timed[-1]
    for s in range(ns):
        h_host[s].copy_(torch.from_numpy(h_of(T_e, s)))
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    es = N * N * 16
    dist.barrier()
    torch.cuda.synchronize(dev)
    ee0.record(stream)
    for s in range(ns):
        check(lib().nedy_buf_upload(ht_e2e[s].h, 0, es, C.c_void_p(h_host.data_ptr() + s * es)))
    step_split(T_e, ht_e2e)
    for s in range(ns):
        base = row_host.data_ptr() + s * row_blocks * es
        check(lib().nedy_gf_download(G[s].h, LES, T_e * (T_e + 1) // 2, T_e + 1, C.c_void_p(base)))
        check(lib().nedy_gf_download(G[s].h, RET, T_e * (T_e + 1) // 2, T_e + 1,
                                     C.c_void_p(base + (T_e + 1) * es)))
        check(lib().nedy_gf_download(G[s].h, TV, T_e * (ntau + 1), ntau + 1,
                                     C.c_void_p(base + 2 * (T_e + 1) * es)))
    ee1.record(stream)
    torch.cuda.synchronize(dev)
    dist.barrier()
    e2e_secs = dist.max(ee0.elapsed_time(ee1) / 1e3)
    h2d = ns * es
    d2h = ns * (2 * (T_e + 1) + ntau + 1) * es
    torch.cuda.synchronize(dev)
    pstats = ctx.predictor_stats() if pred is not None else None
    rep = C.create_string_buffer(16384)
    check(lib().nedy_split_tune_report(rep, 16384))
    tune = [x for x in rep.value.decode().split(";") if x]
    return dict(plain=plain, split=split, split_iters=split_iters, max_dg=max_dg, err=err, max_g=max_g, T=T_timed,
                e2e_secs=e2e_secs, h2d=h2d, d2h=d2h, prep=prep, pred_info=pred_info, pred_stats=pstats, tune=tune,
                mu=list(mus))


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
                       f"pre-evolved {args.state} state; plain form {args.corr} corrector iterations in FP64, split form "
                       f"split-precision self-energy with the residual exit at {args.tol:g} (at most {args.corr})",
           "nao": args.nao, "naux": args.naux, "ntau": args.ntau, "nspin": 1 if args.restricted else 2, "t_window": [args.t0 + W, args.t0 + W + K - 1],
           "corr_steps": args.corr, "precision": "fp64", "predictor": "polynomial extrapolation (k=5)",
           "l2": "inputs (G, Sigma histories) larger than L2; no flush needed",
           "parallelism": f"replicas x{dist.world}"}
    if args.impl == "reference":
        if dist.rank != 0:
            dist.close()
            return
        samples = []
        for i in range(W + K):
            smp = cpu_sample(args)
            if i >= W:
                samples.append(smp)
        T_mid = args.t0 + W
        step_s = float(np.mean([cpu_step_seconds(s, T_mid, args) for s in samples]))
        value = 1.0 / step_s
        line = {"metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": 0, "steps": K, "warmup": W,
                "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "complex128", "data": "synthetic (seeded)", "config": cfg, "impl": "reference",
                "cpu_baseline": cpu_baseline_obj(samples[-1], value, args),
                "e2e": {"value": value, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        dist.close()
        return

    fp64 = fp64_gemm_peak(dist.local) if dist.rank == 0 else None
    r = run_engine(args, dist)
    sp, pl = r["split"], r["plain"]
    value = replica_value(K, dist.world, sp["secs"])
    plain_value = replica_value(K, dist.world, pl["secs"]) if pl else None
    T_mid = r["T"][len(r["T"]) // 2]
    peaks, src = measured_peaks()
    cfg["precision"] = ({"bf16x2": "split self-energy, two BF16 pieces per operand, products hi*hi + hi*lo + lo*hi",
                         "bf16x3": "split self-energy, three BF16 pieces per operand, six products"}[args.split_mode] +
                        " (tcgen05, FP32 accumulation), FP64 Dyson/HF/density; plain form FP64 throughout")
    cfg["predictor"] = ("learned MLP correction of the k=5 extrapolation (polynomial fallback)" if args.predictor == "learned"
                        else "polynomial extrapolation (k=5)") + " + residual exit at max|dG| estimate <= tol"
    cfg["state"] = (f"GF2 trajectory from the {'restricted' if args.restricted else 'unrestricted'} HF equilibrium "
                    "(Gaussian pulse E0=0.05 t0=2 sigma=0.5)"
                    if args.state == "trajectory" else "synthetic free-propagation history, 0.1 sin(2t) drive")
    cfg["tol"] = args.tol
    line = {"metric": METRIC, "value": value, "unit": "timesteps/s", "n_gpus": dist.world, "steps": K, "warmup": W,
            "ms_per_step": sp["secs"] / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "complex128 state; self-energy contractions in BF16 pieces with FP32 accumulation",
            "data": ("synthetic (seeded random h0, B^Q, dipole); state: " + cfg["state"]), "config": cfg}
    if dist.rank == 0:
        # dominant kernel of the headline form: the split GEMM (BF16 piece products on tcgen05);
        # achieved = algorithmic BF16 pipe FLOPs / its summed device time (CUDA events per launch)
        bf16_peak = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
        ach = sp["split_flops"] / (sp["split_ms"] / 1e3) / 1e12 if sp.get("split_ms") else None
        sig_flops = sum(flops_sigma(t, args.nao, args.naux, args.ntau, 1 if args.restricted else 2)
                        for t in r["T"]) * args.corr
        peak_key = "bf16_tflops_sustained" if peaks.get("bf16_tflops_sustained") else "bf16_tflops"
        # DRAM traffic of the split GEMMs per step: bytes per exchange unit (one slice of one
        # spin; dram__bytes_read.sum + dram__bytes_write.sum of every split GEMM class, ncu
        # capture of the nao=64, naux=256, ntau=32 case with two pieces per operand, S' and Q
        # dominating at 134 MB and 192 MB) times the units of the step (les, tv and ret slices)
        ns = 1 if args.restricted else 2
        units = sum(ns * (2 * (t + 1) + args.ntau + 1) * it for t, it in zip(r["T"], r["split_iters"])) / K
        per_unit = 3.6e8 if (args.nao, args.naux, args.split_mode) == (64, 256, "bf16x2") else None
        line["roofline"] = {"bound": "tensor", "kernel": "split_gemm_kernel (BF16 piece products, tcgen05, TMEM)",
                            "achieved": ach, "peak": bf16_peak, "unit": "TFLOP/s",
                            "frac": (ach / bf16_peak) if ach else None,
                            "traffic": per_unit * units if per_unit else None,
                            "traffic_unit": "bytes per step (DRAM, all split GEMM launches of one step)",
                            "exchange_units_per_step": units,
                            "peak_source": f"{src}: {peak_key} (kernel timed inside a long step)",
                            "algorithmic_flops_per_step": sp["split_flops"] / K,
                            "kernel_ms_per_step": sp["split_ms"] / K}
        line["forms"] = {
            "split_predictor": {"timesteps_s": value, "ms_per_step": sp["secs"] / K * 1e3,
                                "iterations_per_step": r["split_iters"],
                                "phase_ms": dict(zip(["predictor", "mean_field", "self_energy", "dyson"], sp["phase_ms"])),
                                "gpu_launches": sp["launches"]},
            "plain_fp64": {"timesteps_s": plain_value, "ms_per_step": pl["secs"] / K * 1e3,
                           "iterations_per_step": args.corr,
                           "phase_ms": dict(zip(["predictor", "mean_field", "self_energy", "dyson"], pl["phase_ms"])),
                           "gpu_launches": pl["launches"],
                           "self_energy_fp64_tflops": sig_flops / (pl["phase_ms"][2] / 1e3) / 1e12,
                           "fp64_peak_tflops": fp64} if pl else None,
            "state_preparation": r["prep"], "predictor_training": r["pred_info"],
            "predictor_stats": r["pred_stats"], "split_tile_autotune": r["tune"],
            "speedup_split_vs_plain": value / plain_value if pl else None,
            "max_abs_dG_split_vs_plain": r["max_dg"], "error_vs_fp64_per_component": r["err"],
            "max_abs_G": r["max_g"], "mu": r["mu"]}
        line["clocks"] = sp["clocks"]
        line["clocks_plain"] = pl["clocks"] if pl else None
        line["gpu_launches"] = sp["launches"]
        line["e2e"] = {"value": dist.world / r["e2e_secs"], "unit": "timesteps/s", "h2d_bytes_per_step": r["h2d"],
                       "d2h_bytes_per_step": r["d2h"]}
        if dist.world == 1 and not args.no_cpu_baseline:
            smp = cpu_sample(args)
            v = 1.0 / cpu_step_seconds(smp, T_mid, args)
            line["cpu_baseline"] = cpu_baseline_obj(smp, v, args)
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
