"""CPU model of the split-precision arithmetic behind the tolerances of the GPU tests.

An FP64 operand is split into BF16 pieces (each the BF16 rounding of what the previous
ones left), the piece products are formed exactly and accumulated in FP32 once per
16-deep K step, as the tcgen05 kernels do.  The model shows (i) two pieces with three
products and three pieces with six products both stay far inside the 1e-4 relative
bound of tests/test_split_gemm.py, and (ii) the FP32 accumulation, not the piece count,
sets the floor, which is why the two-piece mode gives the same G as the three-piece one
within the residual-exit tolerance.
"""
import numpy as np
import pytest
import torch

PRODUCTS = {2: [(0, 0), (0, 1), (1, 0)], 3: [(0, 0), (0, 1), (1, 0), (0, 2), (1, 1), (2, 0)]}


def pieces(x, n):
    out, r = [], x.copy()
    for _ in range(n):
        h = torch.from_numpy(r).to(torch.bfloat16).to(torch.float64).numpy()
        out.append(h)
        r = r - h
    return out


def split_gemm_model(a, b, n):
    A, B = pieces(a, n), pieces(b, n)
    M, K = a.shape
    acc = np.zeros((M, b.shape[0]), np.float32)
    for k0 in range(0, K, 16):
        blk = sum(A[i][:, k0:k0 + 16] @ B[j][:, k0:k0 + 16].T for i, j in PRODUCTS[n])
        acc = (acc + blk.astype(np.float32)).astype(np.float32)
    return acc.astype(np.float64)


@pytest.mark.parametrize("K", [256, 1024])
def test_piece_products_with_fp32_accumulation(K):
    rng = np.random.default_rng(K)
    a = rng.uniform(-1, 1, (48, K))
    b = rng.uniform(-1, 1, (40, K))
    ref = a @ b.T
    err = {n: np.abs(split_gemm_model(a, b, n) - ref).max() / np.abs(ref).max() for n in (2, 3)}
    assert err[2] < 2e-5 and err[3] < 2e-5      # well inside the 1e-4 bound of the GPU checks
    assert err[3] <= err[2]                      # more pieces never hurt
    # the pieces alone (exact accumulation) would be far more accurate than FP32 allows
    A2, B2 = pieces(a, 2), pieces(b, 2)
    exact2 = sum(A2[i] @ B2[j].T for i, j in PRODUCTS[2])
    assert np.abs(exact2 - ref).max() / np.abs(ref).max() < 1e-4


def test_pieces_represent_operands():
    x = np.random.default_rng(1).uniform(-1e3, 1e3, 4096)
    for n, bound in ((1, 2.0 ** -8), (2, 2.0 ** -16), (3, 2.0 ** -24)):
        rel = np.abs(sum(pieces(x, n)) - x) / np.abs(x)
        assert rel.max() <= bound
