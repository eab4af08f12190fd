"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is the C++ restatement of the reference solver in this directory.
Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use it, and there only as the checker / timed CPU baseline.

Green's functions are passed as any object with the attributes of
``nedyson_b200.greens.HostGF`` (nt, ntau, nao, sig and C-contiguous complex128
arrays les, ret, tv, mat).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


class _GF(C.Structure):
    _fields_ = [("nt", C.c_int), ("ntau", C.c_int), ("nao", C.c_int), ("sig", C.c_int),
                ("les", C.c_void_p), ("ret", C.c_void_p), ("tv", C.c_void_p), ("mat", C.c_void_p)]


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def _find_blas():
    try:
        import scipy
    except Exception:
        return None
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if f.startswith("libscipy_openblas") and "64_" not in f and f.endswith(".so"):
            return os.path.join(d, f)
    return None


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    L = C.CDLL(LIB)
    P, D, I = C.c_void_p, C.c_double, C.c_int
    sig = {
        "orc_set_blas": ([C.c_char_p, I], I), "orc_have_blas": ([], I), "orc_set_threads": ([I], None),
        "orc_get_threads": ([], I),
        "orc_integrator_tables": ([I, P, P, P, P, P, P, P], None), "orc_gregory_weight": ([I, I, I], D),
        "orc_colloc_nodes": ([I, P, P], None),
        "orc_dyson_new": ([I, I, I, I], P), "orc_dyson_free": ([P], None),
        "orc_mixing": ([P, P, P, P, D, D], None), "orc_mixing_kernel": ([P, P, P, D, D], None),
        "orc_lesser": ([P, P, P, P, D], None), "orc_energy": ([P, P, P, D, D, P], None),
        "orc_extrapolate": ([P, I, P], None), "orc_ctv1": ([P, P, P, P, P, I, D], None),
        "orc_ctv_tstp": ([P, I, P, P, P, P, P, D, D], None),
        "orc_cles2": ([P, P, P, P, P, I, D, P], None), "orc_cles3": ([P, P, P, P, P, I, D, P], None),
        "orc_energy_conv": ([P, I, P, P, D, D], D),
        "orc_dyson_step": ([P, I, P, P, P, D, D, D, P], D), "orc_dyson_start": ([P, P, P, P, D, D, D], D),
        "orc_g0_from_h0": ([P, P, D, P, D, D], None), "orc_herm_eig": ([I, P, P, P], None),
        "orc_df_new": ([I, I, P, P], P), "orc_df_free": ([P], None),
        "orc_df_solve": ([P, I, P, P], None), "orc_df_solve_loop": ([P, I, P, P], None),
        "orc_df_solve_spin": ([P, I, P, P], None), "orc_df_solve_spin_loop": ([P, I, P, P], None),
        "orc_df_solve_spin_jobs": ([P, I, P, P, I, I], None), "orc_df_solve_jobs": ([P, I, P, P, I, I], None),
        "orc_full_new": ([I, P, P], P), "orc_full_free": ([P], None),
        "orc_full_solve": ([P, I, P, P], None), "orc_full_solve_loop": ([P, I, P, P], None),
        "orc_hf_decomp": ([I, I, P, P, P], None), "orc_hf_decomp_loop": ([I, I, P, P, P], None),
        "orc_hf_spin_decomp": ([I, I, P, P, P, P], None), "orc_hf_spin_decomp_loop": ([I, I, P, P, P, P], None),
        "orc_hf_full": ([I, P, P, P], None), "orc_hf_full_loop": ([I, P, P, P], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    blas = os.environ.get("NEDY_ORACLE_BLAS") or _find_blas()
    if blas and os.environ.get("NEDY_ORACLE_NOBLAS") != "1":
        L.orc_set_blas(blas.encode(), 1)
    _lib = L
    return L


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def gf(g) -> _GF:
    for a in (g.les, g.ret, g.tv, g.mat):
        assert a.dtype == np.complex128 and a.flags.c_contiguous
    return _GF(g.nt, g.ntau, g.nao, g.sig, _p(g.les), _p(g.ret), _p(g.tv), _p(g.mat))


def gf_pair(a, b):
    arr = (_GF * 2)(gf(a), gf(b))
    return arr


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


def integrator_tables(k: int):
    k1 = k + 1
    out = dict(poly_interp=np.zeros(k1 * k1), poly_diff=np.zeros(k1 * k1), poly_integ=np.zeros(k1 ** 3),
               bd=np.zeros(k1 + 1), start=np.zeros(k1 * k1), Omega=np.zeros(k1 * k1), ex=np.zeros(k1))
    lib().orc_integrator_tables(k, *[_p(out[n]) for n in ("poly_interp", "poly_diff", "poly_integ", "bd",
                                                           "start", "Omega", "ex")])
    return out


def gregory_weight(k: int, n: int, j: int) -> float:
    return lib().orc_gregory_weight(k, n, j)


def colloc_nodes(ntau: int):
    x = np.zeros(ntau + 1)
    w = np.zeros(ntau + 1)
    lib().orc_colloc_nodes(ntau, _p(x), _p(w))
    return x, w


class Dyson:
    """Oracle counterpart of NEdyson::dyson (reference src/dyson.h:17-143)."""

    def __init__(self, nt, ntau, nao, k=5):
        self.nt, self.ntau, self.nao, self.k = nt, ntau, nao, k
        self.h = lib().orc_dyson_new(nt, ntau, nao, k)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_dyson_free(self.h)
            self.h = None

    def mixing(self, A, B, beta, sig):
        res = np.zeros((self.ntau + 1, self.nao, self.nao), np.complex128)
        lib().orc_mixing(self.h, _p(res), _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)), beta, sig)
        return res

    def mixing_kernel(self, B, beta, sig):
        np1 = self.ntau + 1
        K = np.zeros((np1, np1, self.nao, self.nao), np.complex128)
        lib().orc_mixing_kernel(self.h, _p(K), _p(np.ascontiguousarray(B)), beta, sig)
        return K

    def lesser(self, A, B, beta):
        res = np.zeros((self.nao, self.nao), np.complex128)
        lib().orc_lesser(self.h, _p(res), _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)), beta)
        return res

    def energy(self, A, B, beta, sig):
        out = np.zeros(2)
        lib().orc_energy(self.h, _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)), beta, sig, _p(out))
        return complex(out[0], out[1])

    def extrapolate(self, n, G):
        lib().orc_extrapolate(self.h, n, C.byref(gf(G)))

    def ctv1(self, A, Acc, B, n, dt):
        res = np.zeros((self.ntau + 1, self.nao, self.nao), np.complex128)
        lib().orc_ctv1(self.h, _p(res), C.byref(gf(A)), C.byref(gf(Acc)), C.byref(gf(B)), n, dt)
        return res

    def ctv_tstp(self, tstp, Cg, A, Acc, B, Bcc, beta, dt):
        lib().orc_ctv_tstp(self.h, tstp, C.byref(gf(Cg)), C.byref(gf(A)), C.byref(gf(Acc)), C.byref(gf(B)),
                           C.byref(gf(Bcc)), beta, dt)

    def cles2(self, A, Acc, B, Bcc, m, dt):
        num = max(m, self.k)
        res = np.zeros((num + 1, self.nao, self.nao), np.complex128)
        lib().orc_cles2(self.h, C.byref(gf(A)), C.byref(gf(Acc)), C.byref(gf(B)), C.byref(gf(Bcc)), m, dt, _p(res))
        return res

    def cles3(self, A, Acc, B, Bcc, m, beta):
        top = max(m, self.k)
        res = np.zeros((top + 1, self.nao, self.nao), np.complex128)
        lib().orc_cles3(self.h, C.byref(gf(A)), C.byref(gf(Acc)), C.byref(gf(B)), C.byref(gf(Bcc)), m, beta,
                        _p(res))
        return res

    def energy_conv(self, tstp, Sig, G, beta, dt):
        return lib().orc_energy_conv(self.h, tstp, C.byref(gf(Sig)), C.byref(gf(G)), beta, dt)

    def dyson_step(self, n, G, Sig, hmf, mu, beta, dt):
        parts = np.zeros(3)
        e = lib().orc_dyson_step(self.h, n, C.byref(gf(G)), C.byref(gf(Sig)), _p(hmf), mu, beta, dt, _p(parts))
        return e, parts

    def dyson_start(self, G, Sig, hmf, mu, beta, dt):
        return lib().orc_dyson_start(self.h, C.byref(gf(G)), C.byref(gf(Sig)), _p(hmf), mu, beta, dt)

    def g0_from_h0(self, G, mu, H0, beta, dt):
        H0 = np.ascontiguousarray(H0, np.float64)
        lib().orc_g0_from_h0(self.h, C.byref(gf(G)), mu, _p(H0), beta, dt)


class DF:
    """Oracle counterpart of molGF2SolverDecomp / molGF2SolverSpinDecomp."""

    def __init__(self, Vija: np.ndarray):
        self.Vija = np.ascontiguousarray(Vija, np.float64)
        self.nao, _, self.naux = Vija.shape
        self.Viaj = np.ascontiguousarray(self.Vija.transpose(0, 2, 1))
        self.h = lib().orc_df_new(self.nao, self.naux, _p(self.Vija), _p(self.Viaj))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_df_free(self.h)
            self.h = None

    def solve(self, tstp, Sig, G):
        lib().orc_df_solve(self.h, tstp, C.byref(gf(Sig)), C.byref(gf(G)))

    def solve_loop(self, tstp, Sig, G):
        lib().orc_df_solve_loop(self.h, tstp, C.byref(gf(Sig)), C.byref(gf(G)))

    def solve_spin(self, tstp, Sig2, G2):
        lib().orc_df_solve_spin(self.h, tstp, gf_pair(*Sig2), gf_pair(*G2))

    def solve_jobs(self, tstp, Sig, G, job_lo, job_hi):
        """Slices [job_lo, job_hi) of the restricted row T (lesser t, then retarded t, then mixed
        tau); Sigma is not zeroed first."""
        lib().orc_df_solve_jobs(self.h, tstp, C.byref(gf(Sig)), C.byref(gf(G)), int(job_lo), int(job_hi))

    def solve_spin_jobs(self, tstp, Sig2, G2, job_lo, job_hi):
        """Slices [job_lo, job_hi) of the unrestricted row T (lesser t, then retarded t, then
        mixed tau; both spins per slice); Sigma is not zeroed first."""
        lib().orc_df_solve_spin_jobs(self.h, tstp, gf_pair(*Sig2), gf_pair(*G2), int(job_lo), int(job_hi))

    def solve_spin_loop(self, tstp, Sig2, G2):
        lib().orc_df_solve_spin_loop(self.h, tstp, gf_pair(*Sig2), gf_pair(*G2))

    def hf(self, hmf_t, rho):
        lib().orc_hf_decomp(self.nao, self.naux, _p(self.Vija), _p(hmf_t), _p(np.ascontiguousarray(rho)))

    def hf_loop(self, hmf_t, rho):
        lib().orc_hf_decomp_loop(self.nao, self.naux, _p(self.Vija), _p(hmf_t), _p(np.ascontiguousarray(rho)))

    def hf_spin(self, h_up, h_dn, rho2):
        lib().orc_hf_spin_decomp(self.nao, self.naux, _p(self.Vija), _p(h_up), _p(h_dn),
                                 _p(np.ascontiguousarray(rho2)))

    def hf_spin_loop(self, h_up, h_dn, rho2):
        lib().orc_hf_spin_decomp_loop(self.nao, self.naux, _p(self.Vija), _p(h_up), _p(h_dn),
                                      _p(np.ascontiguousarray(rho2)))


class Full:
    """Oracle counterpart of molGF2Solver (full U)."""

    def __init__(self, U: np.ndarray, Uexch: np.ndarray):
        self.U = np.ascontiguousarray(U, np.float64)
        self.Uexch = np.ascontiguousarray(Uexch, np.float64)
        self.nao = U.shape[0]
        self.h = lib().orc_full_new(self.nao, _p(self.U), _p(self.Uexch))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_full_free(self.h)
            self.h = None

    def solve(self, tstp, Sig, G):
        lib().orc_full_solve(self.h, tstp, C.byref(gf(Sig)), C.byref(gf(G)))

    def solve_loop(self, tstp, Sig, G):
        lib().orc_full_solve_loop(self.h, tstp, C.byref(gf(Sig)), C.byref(gf(G)))

    def hf(self, hmf_t, rho):
        lib().orc_hf_full(self.nao, _p(self.U), _p(hmf_t), _p(np.ascontiguousarray(rho)))

    def hf_loop(self, hmf_t, rho):
        lib().orc_hf_full_loop(self.nao, _p(self.U), _p(hmf_t), _p(np.ascontiguousarray(rho)))
