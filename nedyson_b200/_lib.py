"""ctypes binding of the engine's C ABI (include/nedy.h).

Loads the in-tree ``libnedy_b200.so``.  There is no fallback: if the library is
missing or cannot be loaded, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libnedy_b200.so")

NEDY_OK = 0
LES, RET, TV, MAT = 0, 1, 2, 3
PREC_FP64, PREC_SPLIT_BF16X3, PREC_SPLIT_BF16X2 = 0, 1, 2


class NedyConfig(C.Structure):
    _fields_ = [("nt", C.c_int), ("ntau", C.c_int), ("nao", C.c_int), ("k", C.c_int),
                ("beta", C.c_double), ("dt", C.c_double), ("device", C.c_int),
                ("workspace_bytes", C.c_longlong)]


class BatchInstance(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("G", C.c_void_p), ("Sigma", C.c_void_p), ("hmf", C.c_void_p),
                ("h_all", C.c_void_p), ("mu", C.c_double)]


class NedyError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"nedy status {status}: {msg}")
        self.status = status


# exported entry points and their signatures: (argtypes, restype)
_P, _I, _D, _LL = C.c_void_p, C.c_int, C.c_double, C.c_longlong
_PP = C.POINTER(C.c_void_p)
_DP = C.POINTER(C.c_double)
SIGNATURES = {
    "nedy_abi_version": ([], _I),
    "nedy_status_string": ([_I], C.c_char_p),
    "nedy_last_error": ([], C.c_char_p),
    "nedy_ctx_create": ([C.POINTER(NedyConfig), _PP], _I),
    "nedy_ctx_destroy": ([_P], _I),
    "nedy_ctx_synchronize": ([_P], _I),
    "nedy_collocation_nodes": ([_P, _DP, _DP], _I),
    "nedy_ctx_stream": ([_P, _PP], _I),
    "nedy_ctx_set_timing": ([_P, _I], _I),
    "nedy_ctx_phase_times": ([_P, _DP], _I),
    "nedy_ctx_inject_split_error": ([_P, _I], _I),
    "nedy_dense_solve": ([_P, _I, _I, _I, _P, _P], _I),
    "nedy_launch_count": ([], C.c_ulonglong),
    "nedy_gf_create": ([_P, _I, _I, _I, _I, _PP], _I),
    "nedy_gf_create_windowed": ([_P, _I, _I, _I, _I, _I, _PP], _I),
    "nedy_gf_window": ([_P, C.POINTER(C.c_int)], _I),
    "nedy_gf_create_host_history": ([_P, _I, _I, _I, _I, _PP], _I),
    "nedy_gf_host_history": ([_P, C.POINTER(C.c_int)], _I),
    "nedy_gf_destroy": ([_P], _I),
    "nedy_gf_upload": ([_P, _I, _LL, _LL, _P], _I),
    "nedy_gf_download": ([_P, _I, _LL, _LL, _P], _I),
    "nedy_gf_device_pointer": ([_P, _I, _PP], _I),
    "nedy_gf_set_tstp_zero": ([_P, _I], _I),
    "nedy_buf_create": ([_P, _LL, _PP], _I),
    "nedy_buf_destroy": ([_P], _I),
    "nedy_buf_upload": ([_P, _LL, _LL, _P], _I),
    "nedy_buf_download": ([_P, _LL, _LL, _P], _I),
    "nedy_buf_device_pointer": ([_P, _PP], _I),
    "nedy_set_df_tensor": ([_P, _P, _I, _I], _I),
    "nedy_set_full_tensor": ([_P, _P, _P, _I], _I),
    "nedy_gf2_decomp_solve": ([_P, _I, _P, _P], _I),
    "nedy_gf2_spin_decomp_solve": ([_P, _I, _P, _P, _P, _P], _I),
    "nedy_gf2_full_solve": ([_P, _I, _P, _P], _I),
    "nedy_get_dm": ([_P, _P, _I, _P, _LL], _I),
    "nedy_hf_decomp": ([_P, _I, _P, _P], _I),
    "nedy_hf_decomp_noalloc": ([_P, _I, _P, _P], _I),
    "nedy_ctx_set_precision": ([_P, _I], _I),
    "nedy_split_stats": ([_I, _DP, _DP], _I),
    "nedy_split_autotune": ([_I], _I),
    "nedy_sigma_chunk_plan": ([_I, _I, _LL, _I, _I, _I, C.POINTER(_I), C.POINTER(_I)], _I),
    "nedy_split_gemm_check": ([_I] * 17 + [C.c_ulonglong, C.POINTER(C.c_double)], _I),
    "nedy_split_tune_report": ([C.c_char_p, _I], _I),
    "nedy_split_tune_pending": ([C.POINTER(C.c_int)], _I),
    "nedy_predictor_create": ([_P, _LL, C.c_ulonglong, _PP], _I),
    "nedy_predictor_destroy": ([_P], _I),
    "nedy_predictor_collect": ([_P, _P, _I, _I], _I),
    "nedy_predictor_samples": ([_P, C.POINTER(_LL)], _I),
    "nedy_predictor_clear": ([_P], _I),
    "nedy_predictor_train": ([_P, _I, _I, _D, _DP], _I),
    "nedy_predictor_nparams": ([], _LL),
    "nedy_predictor_params": ([_P, _P, _I], _I),
    "nedy_predictor_forward": ([_P, _P, _I, _P], _I),
    "nedy_predictor_infer": ([_P, _P, _I, _P], _I),
    "nedy_predictor_loss_grad": ([_P, _P, _P, _I, _DP, _P], _I),
    "nedy_predict": ([_P, _I, _P, _I], _I),
    "nedy_ctx_set_predictor": ([_P, _P], _I),
    "nedy_ctx_predictor_stats": ([_P, C.POINTER(_I), C.POINTER(_LL), C.POINTER(_LL), _DP], _I),
    "nedy_decomp_spin_tstp_tol": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double, _I, C.c_double,
                                   C.POINTER(_I), C.POINTER(C.c_double)], _I),
    "nedy_decomp_tstp_tol": ([_P, _I, _P, _P, _P, _P, C.c_double, _I, C.c_double, C.POINTER(_I), C.POINTER(C.c_double)], _I),
    "nedy_hf_spin_decomp": ([_P, _I, _P, _P, _P], _I),
    "nedy_hf_full": ([_P, _I, _P, _P], _I),
    "nedy_extrapolate": ([_P, _I, _P], _I),
    "nedy_dyson_step": ([_P, _I, _P, _P, _P, _D, _DP], _I),
    "nedy_dyson_start": ([_P, _P, _P, _P, _D, _DP], _I),
    "nedy_energy_conv": ([_P, _I, _P, _P, _DP], _I),
    "nedy_decomp_tstp": ([_P, _I, _P, _P, _P, _P, _D, _I, _DP], _I),
    "nedy_full_tstp": ([_P, _I, _P, _P, _P, _P, _D, _I, _DP], _I),
    "nedy_matsubara_gf2": ([_P, _I, _PP, _PP, _PP, _PP, _PP, _D, _I, _D, C.POINTER(_I), _DP], _I),
    "nedy_batch_create": ([C.POINTER(BatchInstance), _I, _I, _PP], _I),
    "nedy_batch_destroy": ([_P], _I),
    "nedy_batch_tstp": ([_P, _I, _I, _D, C.POINTER(_I)], _I),
    "nedy_decomp_spin_tstp": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _I, _DP], _I),
}

_lib = None


def lib():
    """The loaded engine library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"engine library not built: {LIBPATH} (run python -m nedyson_b200.build)")
        L = C.CDLL(LIBPATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(status: int):
    if status != NEDY_OK:
        msg = lib().nedy_last_error()
        raise NedyError(status, msg.decode() if msg else lib().nedy_status_string(status).decode())
