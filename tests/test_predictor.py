"""Learned next-step predictor: kernels against the CPU restatement, training, ablation.

The network has no counterpart in the reference (whose predictor is the polynomial
extrapolation of dyson::Extrapolate, src/dyson.cpp:47-117).  Its forward pass and
gradients on the GPU are checked against oracle/mlp.py (BF16 operand rounding
emulated, FP64 accumulation): forward within 2e-3 and gradient within 1e-3 of the
largest element.  The ablation trains on trajectories the engine generates and
compares the prediction error with and without the network on a held-out run.
"""
import numpy as np
import pytest

from oracle import mlp


def test_cpu_restatement_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.normal(size=mlp.NPARAM) * 0.1
    x = rng.normal(size=(5, mlp.IN))
    t = rng.normal(size=(5, 2))
    _, g = mlp.loss_grad(p, x, t, rounding=False)
    eps = 1e-6
    for i in rng.choice(mlp.NPARAM, 25, replace=False):
        pp = p.copy()
        pp[i] += eps
        lp, _ = mlp.loss_grad(pp, x, t, rounding=False)
        pp[i] -= 2 * eps
        lm, _ = mlp.loss_grad(pp, x, t, rounding=False)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-7 * max(1.0, abs(g).max())


@pytest.mark.gpu
def test_predictor_forward_and_gradient_match_cpu():
    from nedyson_b200 import api
    ctx = api.Context(12, 8, 4, 5, 1.0, 0.02)
    pr = api.Predictor(ctx, 1 << 10, seed=3)
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (96, mlp.IN)).astype(np.float32)
    t = rng.uniform(-1, 1, (96, 2)).astype(np.float32)
    w = pr.params()
    assert w.size == mlp.NPARAM
    y = pr.forward(x)
    yc, _ = mlp.forward(w, x)
    assert np.abs(y - yc).max() <= 2e-3 * np.abs(yc).max()
    lg, gg = pr.loss_grad(x, t)
    lc, gc = mlp.loss_grad(w, x, t)
    assert abs(lg - lc) <= 1e-4 * abs(lc)
    assert np.abs(gg - gc).max() <= 1e-3 * np.abs(gc).max()
    pr.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 300, 5000])
def test_tensor_core_inference_matches_cpu(n):
    """The inference kernel of the steps (tcgen05, 128 rows per CTA, ragged last tile, more
    tiles than CTAs) against the CPU restatement with the same BF16 operand rounding."""
    from nedyson_b200 import api
    ctx = api.Context(12, 8, 4, 5, 1.0, 0.02)
    pr = api.Predictor(ctx, 1 << 10, seed=7)
    rng = np.random.default_rng(n)
    w = pr.params()
    w += rng.normal(0, 0.05, w.size).astype(np.float32)  # biases and all weights nonzero
    pr.set_params(w)
    x = rng.uniform(-1, 1, (n, mlp.IN)).astype(np.float32)
    y = pr.infer(x)
    yc, _ = mlp.forward(w, x)
    err = np.abs(y - yc).max() / np.abs(yc).max()
    print(f"tensor-core inference n={n}: {err:.2e} of the largest output")
    assert err <= 2e-3
    pr.close()
    ctx.close()


def _sim(seed, kw, nt=50, nao=6):
    from nedyson_b200.inputs import make_problem
    from nedyson_b200.simulation import DecompSimulation
    return DecompSimulation(make_problem(nao, 3 * nao, seed), nt, 24, 10.0, 0.02, drive_kind="gauss", drive_kw=kw)


def _rows(s, t):
    return np.concatenate([s.G.tv_row(t).ravel(), s.G.ret_row(t).ravel(), s.G.les_col(t).ravel()])


@pytest.mark.gpu
def test_predictor_trains_on_engine_trajectories_and_beats_extrapolation():
    from nedyson_b200 import api
    from nedyson_b200._lib import LES, RET, TV, check, lib
    w = None
    losses = []
    for seed, kw in [(11, {"E0": 0.1, "t0": 0.4, "sigma": 0.15}), (14, {"E0": 0.08, "t0": 0.35, "sigma": 0.08})]:
        s = _sim(seed, kw)
        s.free_gf()
        s.do_boot()
        P = api.Predictor(s.ctx, 1 << 21, seed=5)
        if w is not None:
            P.set_params(w)
        for t in range(6, s.nt + 1):
            s.do_tstp_tol(t, 1e-13, 8)
            if t >= 9:
                P.collect(s.G, t, 1)
        assert P.samples() > 10000
        l0 = P.train(1, 1024, 1e-3)
        l1 = P.train(1500, 1024, 1e-3)
        losses.append((l0, l1))
        w = P.params()
        P.close()
        s.ctx.close()
    assert losses[0][1] < 0.5 * losses[0][0]  # training reduces the loss
    # held-out trajectory: prediction errors of the polynomial and the learned predictor
    s = _sim(99, {"E0": 0.07, "t0": 0.45, "sigma": 0.12})
    s.free_gf()
    s.do_boot()
    P = api.Predictor(s.ctx, 1 << 10, seed=5)
    P.set_params(w)
    rms = {0: [], 1: []}
    for t in range(6, s.nt + 1):
        s.do_tstp_tol(t, 1e-13, 8)
        if t in (30, 40, 50):
            conv = _rows(s, t)
            s.ctx.set_predictor(P)
            for learned in (0, 1):
                check(lib().nedy_predict(s.ctx.h, t, s.G.h, learned))
                e = np.abs(_rows(s, t) - conv)
                rms[learned].append(np.sqrt(np.mean(e * e)))
            s.ctx.set_predictor(None)
            nb, N = s.ntau + 1, s.p.nao
            s.G.upload(TV, t * nb, conv[:nb * N * N])
            s.G.upload(RET, t * (t + 1) // 2, conv[nb * N * N:(nb + t + 1) * N * N])
            s.G.upload(LES, t * (t + 1) // 2, conv[(nb + t + 1) * N * N:])
    gain = np.array(rms[0]) / np.array(rms[1])
    print("rms prediction error, polynomial / learned:", gain)
    assert np.all(gain > 1.0)
    P.close()
    s.ctx.close()


@pytest.mark.gpu
def test_learned_predictor_needs_fewer_iterations_at_tight_tolerance():
    """Trained on the first 50 steps of a trajectory (nao=16), the learned prediction beats
    the polynomial one on the judged steps of the next 40 and, at tol 1e-9 where the
    prediction error decides the corrector's iteration count, needs fewer iterations:
    two identical simulations step from the same state, one per predictor."""
    from nedyson_b200 import api
    kw = {"E0": 0.08, "t0": 0.6, "sigma": 0.2}
    sims = [_sim(21, kw, nt=90, nao=16) for _ in range(2)]
    for s in sims:
        s.free_gf()
        s.do_boot()
    P = api.Predictor(sims[0].ctx, 1 << 21, seed=5)
    for t in range(6, 51):
        for s in sims:
            s.do_tstp_tol(t, 1e-13, 8)
        if t >= 9:
            P.collect(sims[0].G, t, 1)
    P.train(2000, 1024, 1e-3)
    sims[0].ctx.set_predictor(P)
    its = [0, 0]
    for t in range(51, 91):
        for i, s in enumerate(sims):
            its[i] += s.do_tstp_tol(t, 1e-9, 6)[0]
    st = sims[0].ctx.predictor_stats()
    print(f"iterations over 40 steps: learned {its[0]}, polynomial {its[1]}; judged {st}")
    assert st["judged"] >= 30 and st["learned_better"] >= 0.8 * st["judged"]
    assert its[0] < its[1]
    P.close()
    for s in sims:
        s.ctx.close()

