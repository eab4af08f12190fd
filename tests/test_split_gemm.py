"""Every instance of the split-precision GEMM (BF16 pieces on tcgen05, FP32 accumulation)
against an FP64 product on seeded operands, through nedy_split_gemm_check.

Tolerance: max |C_split - C_fp64| <= 1e-4 * max |C_fp64| (uniform [-1, 1) operands).
The pieces represent each operand to 2^-24 (three pieces) or 2^-17 (two) relative;
the FP32 accumulation over the K range of one tile dominates: its worst-case bound
K 2^-24 is 6e-5 at K = 1024 (measured 4e-6 .. 1.5e-5, larger for the instances that
split K less).  A layout or descriptor error gives O(1) errors.
"""
import ctypes as C

import pytest

from nedyson_b200 import _lib

pytestmark = pytest.mark.gpu

NEDY_OK, NEDY_ERR_ARG = 0, 1
TOL = {2: 1e-4, 3: 1e-4}

# (M, N, K, nb, a_cplx, b_cplx, conj_a, conj_b, out_pieces, accumulate)
SHAPES = {
    "rxc_pieces": (256, 512, 256, 2, 0, 1, 0, 0, 1, 0),     # one N = 2 BN product per piece pair
    "rxc_conjB_pieces": (256, 384, 192, 2, 0, 1, 0, 1, 1, 0),  # conjugated B: two products; ragged N
    "cxc_acc": (384, 256, 1024, 2, 1, 1, 0, 0, 0, 1),      # FP64 accumulation with a K split
    "cxr_conjA": (256, 320, 128, 1, 1, 0, 1, 0, 0, 0),     # complex x real, ragged last tile
    "cxc_n64_acc": (64, 64, 2048, 3, 1, 1, 0, 1, 0, 1),    # one 64-wide tile per batch
    "cxc_overwrite": (384, 256, 1024, 2, 1, 1, 0, 0, 0, 2),  # replaces C unread (cleared first under a K split)
    "rxc_overwrite": (256, 320, 512, 2, 0, 1, 0, 0, 0, 2),   # ragged last tile
}
# (tile_n, stages, k_block, kdiv, persistent); k_block 0: per-product kernel, 32 / 64: one-load
# kernel; persistent 1: the one-load kernel with one CTA per SM over a tile list and two TMEM
# accumulators (the epilogue of one tile beside the MMAs of the next; 64- or 128-wide tiles),
# BF16 piece outputs only;
# persistent 2: the CTA-pair one-load kernel (tcgen05.mma.cta_group::2, 256-row tiles over
# two CTAs, each staging half of B), complex x complex products only; persistent 3: the
# persistent CTA-pair kernel (clusters of two over a tile list, two accumulators per CTA),
# BF16 piece outputs only
INSTANCES = [(64, 4, 0, 1, 0), (64, 4, 0, 2, 0), (64, 4, 0, 4, 0), (64, 2, 0, 1, 0), (64, 2, 0, 2, 0), (128, 2, 0, 1, 0),
             (128, 3, 0, 1, 0), (128, 4, 0, 1, 0), (256, 2, 0, 1, 0), (256, 3, 0, 1, 0), (256, 2, 0, 2, 0),
             (128, 2, 32, 1, 0), (128, 3, 32, 1, 0), (128, 4, 32, 1, 0), (256, 2, 32, 1, 0), (256, 3, 32, 1, 0),
             (256, 2, 32, 2, 0), (128, 2, 64, 1, 0), (128, 3, 64, 1, 0),
             (128, 2, 32, 1, 1), (128, 3, 32, 1, 1), (128, 4, 32, 1, 1), (128, 2, 64, 1, 1), (128, 2, 32, 2, 1),
             (256, 2, 32, 1, 2), (256, 3, 32, 1, 2), (256, 3, 32, 2, 2), (128, 2, 32, 1, 2), (128, 3, 32, 1, 2),
             (128, 4, 32, 1, 2), (128, 2, 64, 1, 2),
             (128, 3, 32, 1, 3), (128, 4, 32, 1, 3), (128, 2, 64, 1, 3), (128, 3, 64, 1, 3),
             (64, 4, 32, 1, 1), (64, 2, 64, 1, 1), (64, 3, 64, 1, 1)]


@pytest.mark.parametrize("np_", [2, 3])
@pytest.mark.parametrize("shape", list(SHAPES))
def test_split_gemm_instances(shape, np_):
    lib = _lib.lib()
    M, N, K, nb, ac, bc, ca, cb, op, acc = SHAPES[shape]
    ran = []
    for (bn, st, bk, kd, ps) in INSTANCES:
        err = C.c_double(-1.0)
        rc = lib.nedy_split_gemm_check(0, M, N, K, nb, ac, bc, ca, cb, np_, op, acc, bn, st, bk, kd, ps, 17,
                                       C.byref(err))
        if rc == NEDY_ERR_ARG:  # instance absent or too large for shared memory
            continue
        assert rc == NEDY_OK, (shape, bn, st, bk, kd, ps, lib.nedy_last_error())
        print(f"{shape} np={np_} {bn}/{st}/bk{bk}/k{kd}{['', '/persistent', '/pair', '/persistent-pair'][ps]}: {err.value:.3e}")
        assert 0.0 < err.value < TOL[np_], (shape, np_, bn, st, bk, kd, ps, err.value)
        ran.append((bn, st, bk, kd, ps))
    assert len(ran) >= 3, ran
    if N > 64:
        assert any(bk for (_, _, bk, _, _) in ran), "no one-load instance ran"
        if op:  # the persistent kernels write piece outputs
            assert any(ps == 1 for (*_, ps) in ran), "no persistent instance ran"
            assert any(ps == 3 for (*_, ps) in ran), "no persistent CTA-pair instance ran"
        if ac and bc:  # CTA pairs for complex x complex products
            assert any(ps == 2 for (*_, ps) in ran), "no CTA-pair instance ran"


def test_split_gemm_check_rejects_missing_instance():
    err = C.c_double()
    rc = _lib.lib().nedy_split_gemm_check(0, 128, 128, 64, 1, 1, 1, 0, 0, 2, 0, 0, 96, 2, 0, 1, 0, 1, C.byref(err))
    assert rc == NEDY_ERR_ARG
    # the persistent kernel exists only as the one-load kernel with 128-wide tiles
    rc = _lib.lib().nedy_split_gemm_check(0, 128, 256, 64, 1, 1, 1, 0, 0, 2, 0, 0, 256, 2, 32, 1, 1, 1, C.byref(err))
    assert rc == NEDY_ERR_ARG
    # ... and writes BF16 piece outputs only (no FP64 output staging beside four stages)
    rc = _lib.lib().nedy_split_gemm_check(0, 128, 256, 64, 1, 0, 1, 0, 0, 2, 0, 0, 128, 2, 32, 1, 1, 1, C.byref(err))
    assert rc == NEDY_ERR_ARG


def test_split_timeout_path_reports_and_recovers():
    """The bounded-wait give-up path without a fault: the context's error word is preset as a
    wait that gave up would set it, so every CTA of the next split launches skips its work.
    The self-energy call must return NEDY_ERR_TIMEOUT, and the call after it (the report
    cleared the word) must run normally and reproduce the first result."""
    import numpy as np
    from nedyson_b200 import api
    from nedyson_b200.greens import HostGF
    rng = np.random.default_rng(5)
    nao, naux, nt, ntau = 8, 24, 3, 4
    V = rng.uniform(-1, 1, (nao, nao, naux)) / np.sqrt(naux)
    V = 0.5 * (V + V.transpose(1, 0, 2))
    G = HostGF(nt, ntau, nao, -1)
    for a in (G.les, G.ret, G.tv, G.mat):
        a[:] = rng.uniform(-1, 1, a.shape) + 1j * rng.uniform(-1, 1, a.shape)
    ctx = api.Context(5, ntau, nao, 5, 1.0, 0.01)
    ctx.set_precision(_lib.PREC_SPLIT_BF16X2)
    Gd = api.green_func(ctx, nt, ntau, nao, -1).from_host(G)
    Sd = api.green_func(ctx, nt, ntau, nao, -1)
    s = api.molGF2SolverDecomp(ctx, V)
    lib = _lib.lib()
    lib.nedy_split_autotune(0)  # one fixed instance per class: the two good calls run the same kernels
    try:
        _timeout_roundtrip(lib, ctx, s, Sd, Gd, nt)
    finally:
        lib.nedy_split_autotune(1)
        ctx.close()


def _timeout_roundtrip(lib, ctx, s, Sd, Gd, nt):
    import numpy as np
    NEDY_ERR_TIMEOUT = 4
    s.solve(nt, Sd, Gd)
    first = Sd.to_host()
    assert lib.nedy_ctx_inject_split_error(ctx.h, 2) == NEDY_OK
    rc = lib.nedy_gf2_decomp_solve(ctx.h, nt, Sd.h, Gd.h)
    assert rc == NEDY_ERR_TIMEOUT, (rc, lib.nedy_last_error())
    assert b"timed out" in lib.nedy_last_error()
    s.solve(nt, Sd, Gd)  # raises if the word were still set
    again = Sd.to_host()
    for comp in ("les", "ret", "tv"):  # equal up to the order of FP64 atomic sums
        a, b = getattr(again, comp), getattr(first, comp)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), comp
