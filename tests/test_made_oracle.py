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


def test_grouped_density_is_normalised_and_group_autoregressive():
    nb, ns, H, G = 3, 8, 16, 4
    params = MD.init_params(nb, ns, H, seed=2)
    rng = np.random.default_rng(9)
    params = [(W, rng.normal(0, 0.3, b.shape).astype(np.float32)) for W, b in params]
    mk = MD.masks(nb, ns, H, groups=G)
    b = rng.choice([-1.0, 1.0], size=(1, nb))
    xs = np.array(list(itertools.product([-1.0, 1.0], repeat=ns)))
    logits, _ = MD.forward(params, mk, np.repeat(b, len(xs), 0), xs, round_bf16=False)
    assert abs(np.exp(MD.log_density(logits, xs)).sum() - 1.0) < 1e-12
    S = ns // G
    for p in range(ns):
        x2 = xs.copy()
        x2[:, (p // S) * S:] = 1.0                      # the logit of p must ignore its own group and later ones
        l2, _ = MD.forward(params, mk, np.repeat(b, len(xs), 0), x2, round_bf16=False)
        assert np.allclose(l2[:, p], logits[:, p])


def test_block_geometry():
    assert sorted(MD.ORDER.tolist()) == list(range(64))
    ip, fp = MD.internal_pairs(), MD.face_pairs()
    assert ip.shape == (144, 2) and fp.shape == (96, 2)
    assert sorted(fp[:, 1].tolist()) == list(range(96))
    # surface spins: corners on 3 faces, edges on 2, face centres on 1
    counts = np.bincount(fp[:, 0], minlength=64)
    assert sorted(np.bincount(counts).tolist()) == [8, 8, 24, 24]
    # groups of four consecutive positions share no bond
    for w in range(16):
        grp = set(range(4 * w, 4 * w + 4))
        assert not any(a in grp and c in grp for a, c in ip)
    # even positions 0..31 share no bond either
    assert not any(a < 32 and c < 32 for a, c in ip)


def test_same_colour_blocks_do_not_touch():
    L = 16
    for c in range(MD.NCOL):
        cover = np.zeros((L, L, L), np.int64)
        bo = MD.boundary_offsets()
        for b in MD.blocks_of_colour(L, c):
            x0, y0, z0 = MD.block_origin(L, int(b))
            cover[z0:z0 + 4, y0:y0 + 4, x0:x0 + 4] += 1
        assert cover.max() == 1
        # a block's boundary lies inside no block of its colour
        inside = cover.astype(bool)
        for b in MD.blocks_of_colour(L, c):
            x0, y0, z0 = MD.block_origin(L, int(b))
            for (dx, dy, dz) in bo:
                assert not inside[(z0 + dz) % L, (y0 + dy) % L, (x0 + dx) % L]


def test_colour_step_keeps_spins_and_accepts_consistently():
    L, R = 8, 3
    rng = np.random.default_rng(4)
    spins = rng.choice([-1, 1], size=(R, L, L, L)).astype(np.int8)
    params = MD.init_params(96, 64, 32, seed=3)
    mk = MD.masks(96, 64, 32, groups=16)
    before = spins.copy()
    out = MD.colour_step(spins, params, mk, np.array([0.2, 0.22, 0.3]), seed=7, rnd=0, colour=5, groups=16)
    blocks = out["blocks"]
    bnd, now = MD.gather(spins, blocks)
    want = np.where(out["accept"][:, None], out["x_new"], out["x_old"]).reshape(R, len(blocks), 64)
    assert np.array_equal(now, want)
    # sites outside the colour's blocks did not move
    moved = before != spins
    mask = np.zeros((L, L, L), bool)
    for b in blocks:
        x0, y0, z0 = MD.block_origin(L, int(b))
        mask[z0:z0 + 4, y0:y0 + 4, x0:x0 + 4] = True
    assert not moved[:, ~mask].any()
    # x' follows its uniforms: +1 iff u < sigmoid(logit)
    sig = 1.0 / (1.0 + np.exp(-out["logits_new"]))
    assert np.array_equal(out["x_new"] > 0, out["u"] < sig)
