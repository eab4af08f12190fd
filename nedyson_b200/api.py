"""Host-side mirror of the reference classes, running on the B200 engine.

Same names, argument meaning and error behaviour as the reference's C++
classes (reference src/greens.h, src/mol2bSolver.h, src/molHFSolver.h,
src/dyson.h); every call goes through the C ABI of ``libnedy_b200.so``.

    ctx  = Context(nt, ntau, nao, k=5, beta=20.0, dt=0.01)
    G    = green_func(ctx, nt, ntau, nao, -1)         # device-resident, packed layout
    S    = green_func(ctx, nt, ntau, nao, -1)
    gf2  = molGF2SolverDecomp(ctx, Vija)              # Vija: (nao, nao, naux) real
    gf2.solve(T, S, G)                                # Sigma row T
    dy   = dyson(ctx)
    dy.dyson_step(T, G, S, hmf, mu)                   # G row T
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import LES, RET, TV, MAT, check, lib
from .greens import HostGF, tri


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class Context:
    """Engine context: sizes of one simulation (dyson(nt, ntau, nao, k)), beta, dt and the device."""

    def __init__(self, nt, ntau, nao, k=5, beta=1.0, dt=0.01, device=0, workspace_bytes=0):
        self.nt, self.ntau, self.nao, self.k = int(nt), int(ntau), int(nao), int(k)
        self.beta, self.dt = float(beta), float(dt)
        self.device = int(device)
        cfg = _lib.NedyConfig(self.nt, self.ntau, self.nao, self.k, self.beta, self.dt, int(device),
                              int(workspace_bytes))
        h = C.c_void_p()
        check(lib().nedy_ctx_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().nedy_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().nedy_ctx_synchronize(self.h))

    def set_precision(self, mode):
        """Self-energy arithmetic: _lib.PREC_FP64 (default), _lib.PREC_SPLIT_BF16X3 or _lib.PREC_SPLIT_BF16X2."""
        check(lib().nedy_ctx_set_precision(self.h, int(mode)))

    def set_predictor(self, pred: "Predictor | None"):
        """Learned predictor for nedy_decomp_tstp_tol (None: polynomial extrapolation)."""
        check(lib().nedy_ctx_set_predictor(self.h, pred.h if pred is not None else None))

    def predictor_stats(self):
        a, j, b = C.c_int(), C.c_longlong(), C.c_longlong()
        last = (C.c_double * 2)()
        check(lib().nedy_ctx_predictor_stats(self.h, C.byref(a), C.byref(j), C.byref(b), last))
        return {"active": bool(a.value), "judged": j.value, "learned_better": b.value, "last": list(last)}

    def collocation(self):
        x = np.zeros(self.ntau + 1)
        w = np.zeros(self.ntau + 1)
        check(lib().nedy_collocation_nodes(self.h, x.ctypes.data_as(C.POINTER(C.c_double)),
                                           w.ctypes.data_as(C.POINTER(C.c_double))))
        return x, w


class green_func:
    """Device-resident contour Green's function (green_func, reference src/greens.h:17-112)."""

    def __init__(self, ctx: Context, nt, ntau, nao, sig=-1, window: int = 0, host_history: bool = False):
        """window > 0: only the last `window` time steps of G^R and G^< on the device
        (nedy_gf_create_windowed); rows are then read and written one time step at a time.
        host_history: the lesser and retarded triangles in pinned host memory that the kernels
        read over the host link (nedy_gf_create_host_history; for a Sigma whose history exceeds
        the device)."""
        self.ctx = ctx
        self.nt, self.ntau, self.nao, self.sig = int(nt), int(ntau), int(nao), int(sig)
        h = C.c_void_p()
        if host_history:
            if window:
                raise ValueError("green_func: a host-resident history is not windowed")
            check(lib().nedy_gf_create_host_history(ctx.h, self.nt, self.ntau, self.nao, self.sig, C.byref(h)))
        elif window:
            check(lib().nedy_gf_create_windowed(ctx.h, self.nt, self.ntau, self.nao, self.sig, int(window),
                                                C.byref(h)))
        else:
            check(lib().nedy_gf_create(ctx.h, self.nt, self.ntau, self.nao, self.sig, C.byref(h)))
        self.h = h
        w = C.c_int()
        check(lib().nedy_gf_window(h, C.byref(w)))
        self.window = w.value
        check(lib().nedy_gf_host_history(h, C.byref(w)))
        self.host_history = bool(w.value)

    def close(self):
        if getattr(self, "h", None):
            lib().nedy_gf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _nblocks(self, comp):
        return {LES: tri(self.nt), RET: tri(self.nt), TV: (self.nt + 1) * (self.ntau + 1), MAT: self.ntau + 1}[comp]

    def upload(self, comp, first, blocks: np.ndarray):
        blocks = np.ascontiguousarray(blocks, np.complex128)
        nb = blocks.size // (self.nao * self.nao)
        check(lib().nedy_gf_upload(self.h, comp, first, nb, _ptr(blocks)))

    def download(self, comp, first, nb) -> np.ndarray:
        out = np.empty((nb, self.nao, self.nao), np.complex128)
        check(lib().nedy_gf_download(self.h, comp, first, nb, _ptr(out)))
        return out

    def from_host(self, g: HostGF):
        assert (g.nt, g.ntau, g.nao, g.sig) == (self.nt, self.ntau, self.nao, self.sig)
        self.upload(LES, 0, g.les)
        self.upload(RET, 0, g.ret)
        self.upload(TV, 0, g.tv)
        self.upload(MAT, 0, g.mat)
        return self

    def to_host(self) -> HostGF:
        g = HostGF(self.nt, self.ntau, self.nao, self.sig)
        g.les[:] = self.download(LES, 0, tri(self.nt))
        g.ret[:] = self.download(RET, 0, tri(self.nt))
        g.tv[:] = self.download(TV, 0, (self.nt + 1) * (self.ntau + 1)).reshape(g.tv.shape)
        g.mat[:] = self.download(MAT, 0, self.ntau + 1)
        return g

    def set_tstp_zero(self, tstp):
        check(lib().nedy_gf_set_tstp_zero(self.h, tstp))

    # time-slice helpers (contiguous ranges of the packed layout)
    def les_col(self, t):
        return self.download(LES, t * (t + 1) // 2, t + 1)

    def ret_row(self, t):
        return self.download(RET, t * (t + 1) // 2, t + 1)

    def tv_row(self, t):
        return self.download(TV, t * (self.ntau + 1), self.ntau + 1)


class DeviceBuffer:
    def __init__(self, ctx: Context, nbytes: int):
        self.ctx = ctx
        self.nbytes = int(nbytes)
        h = C.c_void_p()
        check(lib().nedy_buf_create(ctx.h, self.nbytes, C.byref(h)))
        self.h = h

    @classmethod
    def from_array(cls, ctx, a: np.ndarray):
        a = np.ascontiguousarray(a)
        b = cls(ctx, a.nbytes)
        b.upload(a)
        return b

    def upload(self, a: np.ndarray, offset: int = 0):
        a = np.ascontiguousarray(a)
        check(lib().nedy_buf_upload(self.h, offset, a.nbytes, _ptr(a)))

    def download(self, shape, dtype=np.complex128, offset: int = 0):
        out = np.empty(shape, dtype)
        check(lib().nedy_buf_download(self.h, offset, out.nbytes, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().nedy_buf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hmf_buffer(ctx: Context, nao: int, hmf: np.ndarray | None = None) -> DeviceBuffer:
    """(nt+1) x nao x nao complex mean-field buffer (the hmf ZTensor<3> of the simulations)."""
    b = DeviceBuffer(ctx, (ctx.nt + 1) * nao * nao * 16)
    if hmf is not None:
        b.upload(np.ascontiguousarray(hmf, np.complex128))
    return b


class molGF2SolverDecomp:
    """Density-fitted restricted GF2 self-energy (reference src/mol2bSolver.h:78-129)."""

    def __init__(self, ctx: Context, Vija: np.ndarray):
        self.ctx = ctx
        self.Vija = np.ascontiguousarray(Vija, np.float64)
        self.nao, _, self.nalpha = self.Vija.shape
        check(lib().nedy_set_df_tensor(ctx.h, _ptr(self.Vija), self.nao, self.nalpha))

    def solve(self, tstp, Sigma: green_func, G: green_func):
        check(lib().nedy_gf2_decomp_solve(self.ctx.h, tstp, Sigma.h, G.h))

    def solve_HF(self, tstp, hmf: DeviceBuffer, rho: DeviceBuffer):
        """molHFSolverDecomp::solve_HF (the GF2 solver derives from the HF solver)."""
        check(lib().nedy_hf_decomp(self.ctx.h, tstp, hmf.h, rho.h))


class molGF2SolverSpinDecomp(molGF2SolverDecomp):
    """Density-fitted unrestricted GF2 self-energy (reference src/mol2bSolver.h:19-71)."""

    def solve(self, tstp, Sigma, G):
        check(lib().nedy_gf2_spin_decomp_solve(self.ctx.h, tstp, Sigma[0].h, Sigma[1].h, G[0].h, G[1].h))

    def solve_HF(self, tstp, hmf, rho2: DeviceBuffer):
        check(lib().nedy_hf_spin_decomp(self.ctx.h, tstp, hmf[0].h, hmf[1].h, rho2.h))


class molGF2Solver:
    """Full-U restricted GF2 self-energy (reference src/mol2bSolver.h:178-209)."""

    def __init__(self, ctx: Context, U: np.ndarray, Uexch: np.ndarray):
        self.ctx = ctx
        self.U = np.ascontiguousarray(U, np.float64)
        self.Uexch = np.ascontiguousarray(Uexch, np.float64)
        self.nao = self.U.shape[0]
        check(lib().nedy_set_full_tensor(ctx.h, _ptr(self.U), _ptr(self.Uexch), self.nao))

    def solve(self, tstp, Sigma, G):
        check(lib().nedy_gf2_full_solve(self.ctx.h, tstp, Sigma.h, G.h))

    def solve_HF(self, tstp, hmf, rho):
        check(lib().nedy_hf_full(self.ctx.h, tstp, hmf.h, rho.h))


class dyson:
    """Dyson-equation machinery (reference src/dyson.h:17-143)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def Extrapolate(self, n, G):
        check(lib().nedy_extrapolate(self.ctx.h, n, G.h))

    def dyson_step(self, n, G, Sig, hmf: DeviceBuffer, mu):
        err = (C.c_double * 3)()
        check(lib().nedy_dyson_step(self.ctx.h, n, G.h, Sig.h, hmf.h, mu, err))
        return float(err[0] + err[1] + err[2]), (err[0], err[1], err[2])

    def dyson_start(self, G, Sig, hmf: DeviceBuffer, mu):
        err = C.c_double()
        check(lib().nedy_dyson_start(self.ctx.h, G.h, Sig.h, hmf.h, mu, C.byref(err)))
        return err.value

    def energy_conv(self, tstp, Sig, G):
        e = C.c_double()
        check(lib().nedy_energy_conv(self.ctx.h, tstp, Sig.h, G.h, C.byref(e)))
        return e.value

    def get_dm(self, G, tstp, rho: DeviceBuffer, offset=0):
        check(lib().nedy_get_dm(self.ctx.h, G.h, tstp, rho.h, offset))


class Predictor:
    """Learned next-step predictor (no reference counterpart; corrects dyson::Extrapolate).

    2-layer MLP of width 256 on the three previous sixth differences of every element's
    time series; trained on the GPU on rows the engine converged."""

    IN = 12

    def __init__(self, ctx: Context, capacity: int = 1 << 22, seed: int = 1):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().nedy_predictor_create(ctx.h, int(capacity), int(seed), C.byref(h)))
        self.h = h
        self.nparams = int(lib().nedy_predictor_nparams())

    def close(self):
        if getattr(self, "h", None):
            lib().nedy_predictor_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def collect(self, G: green_func, tstp: int, stride: int = 1):
        check(lib().nedy_predictor_collect(self.h, G.h, int(tstp), int(stride)))

    def samples(self) -> int:
        n = C.c_longlong()
        check(lib().nedy_predictor_samples(self.h, C.byref(n)))
        return n.value

    def clear(self):
        check(lib().nedy_predictor_clear(self.h))

    def train(self, iters: int, batch: int = 512, lr: float = 1e-3) -> float:
        loss = C.c_double()
        check(lib().nedy_predictor_train(self.h, int(iters), int(batch), float(lr), C.byref(loss)))
        return loss.value

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, np.float32)
        check(lib().nedy_predictor_params(self.h, _ptr(out), 1))
        return out

    def set_params(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.nparams
        check(lib().nedy_predictor_params(self.h, _ptr(w), 0))

    def infer(self, x: np.ndarray) -> np.ndarray:
        """The network through the tensor-core inference kernel (what the steps run)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((x.shape[0], 2), np.float32)
        check(lib().nedy_predictor_infer(self.h, _ptr(x), x.shape[0], _ptr(y)))
        return y

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((x.shape[0], 2), np.float32)
        check(lib().nedy_predictor_forward(self.h, _ptr(x), x.shape[0], _ptr(y)))
        return y

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.empty(self.nparams, np.float32)
        loss = C.c_double()
        check(lib().nedy_predictor_loss_grad(self.h, _ptr(x), _ptr(t), x.shape[0], C.byref(loss), _ptr(g)))
        return loss.value, g
