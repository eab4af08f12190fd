"""The C-ABI library loads and exports every entry point declared in include/nedy.h.

No compute call is made here (no GPU needed); the compute paths are covered by
the gpu-marked parity tests.
"""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nedy.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|unsigned long long|long long)\s*(nedy_\w+)\s*\(", src, re.M)))


@pytest.fixture(scope="module")
def libpath():
    from nedyson_b200 import build
    return build.build()


def test_header_declares_entry_points():
    names = declared()
    assert "nedy_gf2_decomp_solve" in names and "nedy_dyson_step" in names and len(names) >= 30


def test_library_exports_every_declared_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (nedy_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_library_loads_and_answers_without_gpu(libpath):
    from nedyson_b200 import _lib
    L = _lib.lib()
    assert L.nedy_abi_version() == 1
    assert L.nedy_status_string(0) == b"ok"
    assert L.nedy_status_string(7) == b"singular matrix"
    # every binding in the Python table resolves
    for name in _lib.SIGNATURES:
        assert hasattr(L, name)


def test_null_arguments_are_rejected_not_crashing(libpath):
    from nedyson_b200 import _lib
    L = _lib.lib()
    assert L.nedy_ctx_create(None, None) == 1  # NEDY_ERR_ARG
    assert b"null" in L.nedy_last_error()
    assert L.nedy_gf_destroy(None) == 0


def test_step_entry_points_reject_null_handles(libpath):
    """The whole-step entry points check their handles before touching a device."""
    import ctypes as C
    from nedyson_b200 import _lib
    L = _lib.lib()
    it = C.c_int()
    e = C.c_double()
    assert L.nedy_decomp_tstp_tol(None, 6, None, None, None, None, 0.0, 5, 1e-8, C.byref(it), None) == 1
    assert L.nedy_decomp_spin_tstp_tol(None, 6, None, None, None, None, None, None, None, None, 0.0, 0.0, 5, 1e-8,
                                       C.byref(it), None) == 1
    assert b"null" in L.nedy_last_error()
    assert L.nedy_decomp_spin_tstp(None, 6, None, None, None, None, None, None, None, None, 0.0, 0.0, 5,
                                   C.byref(e)) == 1
    assert L.nedy_ctx_set_precision(None, 2) == 1


def test_new_entry_points_reject_bad_arguments(libpath):
    """Full-U step, batch, Matsubara solver, dense solve and the error hook check their
    arguments before touching a device."""
    import ctypes as C
    from nedyson_b200 import _lib
    L = _lib.lib()
    e = C.c_double()
    assert L.nedy_full_tstp(None, 6, None, None, None, None, 0.0, 5, C.byref(e)) == 1
    out = C.c_void_p()
    assert L.nedy_batch_create(None, 0, 0, C.byref(out)) == 1
    inst = (_lib.BatchInstance * 1)()
    assert L.nedy_batch_create(inst, 1, 0, C.byref(out)) == 1  # null handles inside
    assert b"instance 0" in L.nedy_last_error()
    assert L.nedy_batch_tstp(None, 6, 1, 0.0, None) == 1
    assert L.nedy_batch_destroy(None) == 0
    arr = (C.c_void_p * 1)()
    assert L.nedy_matsubara_gf2(None, 1, arr, arr, arr, arr, arr, 1.0, 10, 1e-12, None, None) == 1
    assert L.nedy_ctx_inject_split_error(None, 2) == 1
    assert L.nedy_dense_solve(None, 4, 1, 1, None, None) == 1


def test_tuner_and_host_history_entry_points_without_gpu(libpath):
    """The tuner's pending-classes query answers without a device (no class has run yet);
    the host-history Green's function and its query reject null handles."""
    import ctypes as C
    from nedyson_b200 import _lib
    L = _lib.lib()
    n = C.c_int(-1)
    assert L.nedy_split_tune_pending(C.byref(n)) == 0 and n.value == 0
    assert L.nedy_split_tune_pending(None) == 1
    out = C.c_void_p()
    assert L.nedy_gf_create_host_history(None, 8, 4, 2, -1, C.byref(out)) == 1
    assert L.nedy_gf_host_history(None, C.byref(n)) == 1
