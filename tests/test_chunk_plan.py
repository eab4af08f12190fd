"""Work partition of the density-fitted self-energy (nedy_sigma_chunk_plan, host
arithmetic only, so it runs without a GPU).

The all-split chain sends `sub` exchange units per launch through the S' and Q
contractions; Q has ceil(nao^2 / 128) row tiles per unit, one CTA each, so `sub` is
chosen to fill whole waves of the SMs, and the slices per chunk are a multiple of
`sub` within the workspace budget.
"""
import ctypes as C
import math

import pytest

from nedyson_b200 import _lib

PREC_FP64, PREC_X3, PREC_X2 = 0, 1, 2
GiB = 1 << 30


def plan(nao, naux, budget, prec, sym=1, sms=148):
    ch, sub = C.c_int(), C.c_int()
    rc = _lib.lib().nedy_sigma_chunk_plan(nao, naux, budget, prec, sym, sms, C.byref(ch), C.byref(sub))
    assert rc == 0, _lib.lib().nedy_last_error()
    return ch.value, sub.value


def pieces_unit_bytes(nao, naux, np_):
    kp = lambda k: (k + 63) // 64 * 64
    es = nao * nao
    return 4 * np_ * (es * kp(es) + es * kp(naux) + nao * kp(nao * naux)) + es * naux * 16


def test_bench_size_fills_whole_waves():
    chunk, sub = plan(64, 256, 8 * GiB, PREC_X2)
    assert sub == 23  # 23 units x 32 Q tiles = 736 CTAs = 4.97 waves of 148 SMs
    assert chunk == 46 and chunk % sub == 0


@pytest.mark.parametrize("budget_gib", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("prec", [PREC_X2, PREC_X3])
def test_split_plan_respects_budget_and_waves(budget_gib, prec):
    budget = budget_gib * GiB
    chunk, sub = plan(64, 256, budget, prec)
    np_ = 2 if prec == PREC_X2 else 3
    assert 1 <= sub <= chunk <= 64 and chunk % sub == 0
    assert sub * pieces_unit_bytes(64, 256, np_) <= budget // 2
    waves = 32 * sub / 148
    best = max((32 * u / 148) / math.ceil(32 * u / 148) for u in range(1, sub + 1))
    assert waves / math.ceil(waves) >= min(0.95, best) - 1e-12


def test_fp64_and_general_plans_are_unchanged_by_the_split_rule():
    # FP64, or B^Q not real symmetric: the slice budget of the FP64 intermediates
    for prec, sym in ((PREC_FP64, 1), (PREC_X2, 0)):
        chunk, sub = plan(64, 256, 8 * GiB, prec, sym)
        assert 1 <= sub <= chunk <= 64 and sub <= 16


def test_tiny_budget_degrades_to_single_units():
    assert plan(64, 256, 64 << 20, PREC_X2) == (1, 1)


def test_bad_arguments_are_rejected():
    ch, sub = C.c_int(), C.c_int()
    assert _lib.lib().nedy_sigma_chunk_plan(0, 256, GiB, PREC_X2, 1, 148, C.byref(ch), C.byref(sub)) != 0
    assert _lib.lib().nedy_sigma_chunk_plan(64, 256, GiB, 7, 1, 148, C.byref(ch), C.byref(sub)) != 0
