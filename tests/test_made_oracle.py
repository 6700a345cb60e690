"""The FP64 oracle of the learned block proposal on the CPU: autoregressive masks, a normalised density, and
gradients that match finite differences."""

from __future__ import annotations

import itertools

import numpy as np

from oracle import made as MD


def _tiny(seed=0):
    nb, ns, H = 5, 6, 12
    params = MD.init_params(nb, ns, H, seed=seed)
    rng = np.random.default_rng(seed + 1)
    params = [(W, rng.normal(0, 0.3, b.shape).astype(np.float32)) for W, b in params]
    return nb, ns, H, params, MD.masks(nb, ns, H)


def test_density_is_normalised_and_autoregressive():
    nb, ns, H, params, mk = _tiny()
    rng = np.random.default_rng(3)
    b = rng.choice([-1.0, 1.0], size=(1, nb))
    xs = np.array(list(itertools.product([-1.0, 1.0], repeat=ns)))
    logits, _ = MD.forward(params, mk, np.repeat(b, len(xs), 0), xs, round_bf16=False)
    q = np.exp(MD.log_density(logits, xs))
    assert abs(q.sum() - 1.0) < 1e-12
    # logit j must not depend on spins j..n-1
    for j in range(ns):
        x2 = xs.copy()
        x2[:, j:] = 1.0
        l2, _ = MD.forward(params, mk, np.repeat(b, len(xs), 0), x2, round_bf16=False)
        assert np.allclose(l2[:, j], logits[:, j])


def test_gradients_match_finite_differences():
    nb, ns, H, params, mk = _tiny(1)
    rng = np.random.default_rng(5)
    b = rng.choice([-1.0, 1.0], size=(7, nb))
    x = rng.choice([-1.0, 1.0], size=(7, ns))
    loss, grads = MD.loss_and_grads(params, mk, b, x, round_bf16=False)
    eps = 1e-6
    for li in range(len(params)):
        W, bias = [p.astype(np.float64) for p in params[li]]
        for (i, j) in [(0, 0), (W.shape[0] - 1, W.shape[1] - 1), (W.shape[0] // 2, W.shape[1] // 3)]:
            if mk[li][i, j] == 0:
                assert grads[li][0][i, j] == 0.0
                continue
            P = [(w.astype(np.float64), c.astype(np.float64)) for w, c in params]
            P[li][0][i, j] += eps
            lp, _ = MD.loss_and_grads(P, mk, b, x, round_bf16=False)
            P[li][0][i, j] -= 2 * eps
            lm, _ = MD.loss_and_grads(P, mk, b, x, round_bf16=False)
            assert abs((lp - lm) / (2 * eps) - grads[li][0][i, j]) < 1e-6
        k = bias.shape[0] // 2
        P = [(w.astype(np.float64), c.astype(np.float64)) for w, c in params]
        P[li][1][k] += eps
        lp, _ = MD.loss_and_grads(P, mk, b, x, round_bf16=False)
        P[li][1][k] -= 2 * eps
        lm, _ = MD.loss_and_grads(P, mk, b, x, round_bf16=False)
        assert abs((lp - lm) / (2 * eps) - grads[li][1][k]) < 1e-6


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38], np.float32)
    r = MD.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0      # 1 + 2^-8 is halfway between bf16 neighbours: ties to even
    assert r[2] == 1.0
    assert r[3] == 1.0 + 2 ** -7
    assert r[4] == -2.5
