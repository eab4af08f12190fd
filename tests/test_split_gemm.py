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
}
# (tile_n, stages, k_block, kdiv); k_block 0: per-product kernel, 32 / 64: one-load kernel
INSTANCES = [(64, 4, 0, 1), (64, 4, 0, 2), (64, 4, 0, 4), (64, 2, 0, 1), (64, 2, 0, 2), (128, 2, 0, 1), (128, 3, 0, 1), (128, 4, 0, 1),
             (256, 2, 0, 1), (256, 3, 0, 1), (256, 2, 0, 2), (128, 2, 32, 1), (128, 3, 32, 1), (128, 4, 32, 1),
             (256, 2, 32, 1), (256, 3, 32, 1), (256, 2, 32, 2), (128, 2, 64, 1), (128, 3, 64, 1)]


@pytest.mark.parametrize("np_", [2, 3])
@pytest.mark.parametrize("shape", list(SHAPES))
def test_split_gemm_instances(shape, np_):
    lib = _lib.lib()
    M, N, K, nb, ac, bc, ca, cb, op, acc = SHAPES[shape]
    ran = []
    for (bn, st, bk, kd) in INSTANCES:
        err = C.c_double(-1.0)
        rc = lib.nedy_split_gemm_check(0, M, N, K, nb, ac, bc, ca, cb, np_, op, acc, bn, st, bk, kd, 17,
                                       C.byref(err))
        if rc == NEDY_ERR_ARG:  # instance absent or too large for shared memory
            continue
        assert rc == NEDY_OK, (shape, bn, st, bk, kd, lib.nedy_last_error())
        print(f"{shape} np={np_} {bn}/{st}/bk{bk}/k{kd}: {err.value:.3e}")
        assert 0.0 < err.value < TOL[np_], (shape, np_, bn, st, bk, kd, err.value)
        ran.append((bn, st, bk, kd))
    assert len(ran) >= 3, ran
    if N > 64:
        assert any(bk for (_, _, bk, _) in ran), "no one-load instance ran"


def test_split_gemm_check_rejects_missing_instance():
    err = C.c_double()
    rc = _lib.lib().nedy_split_gemm_check(0, 128, 128, 64, 1, 1, 1, 0, 0, 2, 0, 0, 96, 2, 0, 1, 1, C.byref(err))
    assert rc == NEDY_ERR_ARG
