"""GPU parity of the learned block proposal against the FP64 oracle (oracle/made.py), through the C ABI.

Forward logits and gradients: bfloat16 weights and activations with FP32 accumulation against the oracle's FP64
arithmetic on the same bfloat16-rounded operands (activations re-rounded to bfloat16 between layers), so
results agree to bfloat16 rounding of single activations: logits within 0.05 (median 2e-3), each gradient
tensor within 3 % relative Frobenius error (the kernels also round the backpropagated gradients to bfloat16).
Colour steps: the energy changes are exact integers, the written lattice is exactly x' where accepted and x
elsewhere, the log-densities agree with the oracle's within 0.05, every drawn spin follows its Philox uniform
against the oracle's probability except where the two lie within 0.02 of each other, and every accept decision
follows the kernel's own recorded ratio. A statistical test checks that learned rounds keep the Boltzmann distribution of the plain chain.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import made as MD

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200 import build
    build.build()


def _random_params(seed, scale=1.0, bias_sd=0.2):
    from spin_colour_kernel_b200 import learned as LP
    rng = np.random.default_rng(seed)
    out = []
    for (W, b) in LP.kaiming_params(seed):
        out.append(((W * scale).astype(np.float32), rng.normal(0, bias_sd, b.shape).astype(np.float32)))
    return out


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    return rng.choice([-1.0, 1.0], size=(n, 96)), rng.choice([-1.0, 1.0], size=(n, 64))


def _to_dev(b, x):
    return torch.from_numpy(np.concatenate([b, x], axis=1)).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("groups", [16, 64])
def test_forward_matches_oracle(groups):
    _need_gpu()
    from spin_colour_kernel_b200.learned import BlockProposal
    params = _random_params(1)
    P = BlockProposal(16, 1, groups=groups, params=params)
    b, x = _inputs(256, 2)
    logits, logq = P.forward(_to_dev(b, x))
    mk = MD.masks(96, 64, 256, groups=groups)
    ref, _ = MD.forward(params, mk, b, x)
    err = np.abs(logits.cpu().numpy() - ref)
    assert err.max() < 0.05 and np.median(err) < 2e-3, (err.max(), np.median(err))
    lq_ref = MD.log_density(ref, x)
    assert np.abs(logq.cpu().numpy() - lq_ref).max() < 0.1


def test_tcgen05_forward_matches_mma_sync_forward():
    """Batches of whole 128-row tiles take the tcgen05 GEMMs (accumulator in tensor memory), others the mma.sync
    kernel: the same rows give the same logits up to FP32 summation order (and the rare bfloat16 rounding tie of
    an activation), and no bounded wait gives up."""
    _need_gpu()
    import ctypes
    from spin_colour_kernel_b200 import _lib as L
    from spin_colour_kernel_b200.learned import BlockProposal
    P = BlockProposal(16, 1, groups=16, params=_random_params(11))
    b, x = _inputs(256, 12)
    X = _to_dev(b, x)
    before = ctypes.c_int64()
    L.check(L.lib().sck_wait_timeouts(ctypes.byref(before)))
    l_umma, _ = P.forward(X)          # 256 rows: tcgen05
    l_sync, _ = P.forward(X[:192])    # 192 rows: mma.sync
    d = np.abs(l_umma[:192].cpu().numpy() - l_sync.cpu().numpy())
    assert np.median(d) < 1e-5 and d.max() < 0.05, (np.median(d), d.max())
    after = ctypes.c_int64()
    L.check(L.lib().sck_wait_timeouts(ctypes.byref(after)))
    assert after.value == before.value


@pytest.mark.parametrize("groups", [16, 64])
def test_gradients_match_oracle(groups):
    _need_gpu()
    from spin_colour_kernel_b200.learned import BlockProposal
    params = _random_params(3)
    P = BlockProposal(16, 1, groups=groups, params=params)
    b, x = _inputs(2048, 4)              # two split-K chunks of the weight gradients
    loss, grads = P.grads(_to_dev(b, x))
    mk = MD.masks(96, 64, 256, groups=groups)
    ref_loss, ref = MD.loss_and_grads(params, mk, b, x)
    assert abs(loss - ref_loss) < 1e-3 * max(1.0, abs(ref_loss))
    for li, ((dW, db), (rW, rb)) in enumerate(zip(grads, ref)):
        rel_w = np.linalg.norm(dW - rW) / np.linalg.norm(rW)
        rel_b = np.linalg.norm(db - rb) / max(np.linalg.norm(rb), 1e-12)
        assert rel_w < 3e-2 and rel_b < 3e-2, (li, rel_w, rel_b)
        assert np.all(dW[mk[li] == 0] == 0)


def test_adam_step_follows_its_formula_and_training_lowers_the_loss():
    _need_gpu()
    from spin_colour_kernel_b200.learned import BlockProposal, flatten
    params = _random_params(5)
    P = BlockProposal(16, 1, groups=16, params=params)
    b, x = _inputs(1024, 6)
    # correlated data: the block copies its -x face pattern, so a trained network beats the untrained one
    x[:, :16] = b[:, :16]
    X = _to_dev(b, x)
    _, g = P.grads(X)
    before = flatten(P.get_params())
    P.train(X, steps=1, batch=1024, lr=1e-3)
    after = flatten(P.get_params())
    gf = flatten(g)
    # first step: bias-corrected moments are g and g^2, so the step is lr g / (|g| + eps); compare where the
    # gradient is clearly non-zero (the training step sums the batch in another order)
    step = 1e-3 * gf / (np.abs(gf) + 1e-8)
    big = np.abs(gf) > 1e-5
    np.testing.assert_allclose(after[big], (before - step)[big], rtol=1e-4, atol=1e-6)
    assert np.all(np.abs(after - before) <= 1e-3 * (1 + 1e-4))
    losses = P.train(X, steps=200, batch=512, lr=2e-3)
    assert losses[-20:].mean() < losses[:5].mean() - 1.0


def _lattice(R, L, seed):
    rng = np.random.default_rng(seed)
    return rng.choice([-1, 1], size=(R, L, L, L)).astype(np.int8)


@pytest.mark.parametrize("groups, L", [(16, 16), (64, 8)])
def test_colour_step_matches_oracle(groups, L):
    _need_gpu()
    from spin_colour_kernel_b200.learned import BlockProposal
    R = 6
    params = _random_params(7, scale=0.15, bias_sd=0.05)   # a near-uniform proposal: many accepts
    P = BlockProposal(L, R, groups=groups, params=params)
    mk = MD.masks(96, 64, 256, groups=groups)
    s0 = _lattice(R, L, 8)
    beta = np.linspace(0.05, 0.4, R).astype(np.float32)
    S = torch.from_numpy(s0).cuda()
    B = torch.from_numpy(beta).cuda()
    acc = torch.zeros(R, dtype=torch.int32, device="cuda")
    rec = P.record_buffer()
    nc = (L // 4) ** 3 // 8
    total_acc = 0
    for colour in (0, 5, 7):
        before = S.cpu().numpy()
        rec.zero_()
        P.colour_step(S, B, colour, seed=11, rnd=3, accepted=acc, record=rec)
        after = S.cpu().numpy()
        xs, lq_new, lq_old, dE, accepted = BlockProposal.parse_record(rec, R, nc)
        blocks = MD.blocks_of_colour(L, colour)
        bnd, cur = MD.gather(before, blocks)
        b2, x2, xn = bnd.reshape(-1, 96), cur.reshape(-1, 64), xs.reshape(-1, 64).astype(np.float64)
        # energies: exact
        ip, fp = MD.internal_pairs(), MD.face_pairs()
        dE_ref = MD.block_energy(xn, b2, ip, fp) - MD.block_energy(x2, b2, ip, fp)
        np.testing.assert_array_equal(dE.reshape(-1), dE_ref)
        # densities of the kernel's own proposal and of the current spins
        ln, _ = MD.forward(params, mk, b2, xn)
        lc, _ = MD.forward(params, mk, b2, x2)
        assert np.abs(lq_new.reshape(-1) - MD.log_density(ln, xn)).max() < 0.05
        assert np.abs(lq_old.reshape(-1) - MD.log_density(lc, x2)).max() < 0.05
        # every drawn spin follows its uniform against the oracle's probability (up to near ties)
        uids = (np.arange(R)[:, None] * (L // 4) ** 3 + blocks[None, :]).reshape(-1)
        u, ua = MD.step_uniforms(11, 3, colour, uids)
        p = 1.0 / (1.0 + np.exp(-ln))
        drawn, want_up = xn > 0, u < p
        tie = np.abs(u - p) < 0.02          # the kernel's probabilities differ from the oracle's by < 0.0125
        assert np.array_equal(drawn[~tie], want_up[~tie])
        assert np.mean(drawn != want_up) < 0.01
        # accept decisions follow the kernel's own recorded ratio (float32, up to exp rounding)
        bet = np.repeat(beta, len(blocks)).astype(np.float32)
        logr = (-bet * dE.reshape(-1).astype(np.float32) + lq_old.reshape(-1) - lq_new.reshape(-1)).astype(np.float32)
        pa = np.exp(np.minimum(logr, np.float32(0)))
        tie_a = np.abs(ua - pa) < 1e-5
        assert np.array_equal(accepted.reshape(-1)[~tie_a], (ua < pa)[~tie_a])
        # the lattice: x' where accepted, x elsewhere, nothing else touched
        want = before.copy()
        MD.scatter(want, blocks, xs.astype(np.int8), accepted)
        np.testing.assert_array_equal(after, want)
        total_acc += int(accepted.sum())
    assert int(acc.sum().item()) == total_acc
    assert 0 < total_acc                      # some proposals are accepted at these temperatures


ROUNDS = 1500


def test_learned_rounds_keep_the_boltzmann_distribution():
    """Plain sweeps alone and plain sweeps interleaved with learned rounds give the same mean energy and |M|, within
    2 sigma (sigma from tau_int of each series), on an 8^3 periodic lattice at T = 4.5115. The network is
    trained briefly on the plain chain's blocks, so proposals are accepted often enough for the MH correction to
    matter."""
    _need_gpu()
    from spin_colour_kernel_b200 import system as sy
    from spin_colour_kernel_b200.learned import BlockProposal
    from spin_colour_kernel_b200.sampler import Sampler
    from spin_colour_kernel_b200 import stats
    L, R, T = 8, 512, 4.5115
    s = sy.ising("sc", L)
    res = {}
    for arm in ("plain", "learned"):
        A = Sampler(s, R, device="cuda", seed=21 if arm == "plain" else 22, packed=False)
        A.set_temperature(torch.full((R,), T))
        S = A.init_spins(seed=3)
        beta = torch.full((R,), 1.0 / T, dtype=torch.float32, device="cuda")
        acc = torch.zeros(R, dtype=torch.int32, device="cuda")
        A.sweep(S, 200)
        P = None
        if arm == "learned":
            P = BlockProposal(L, R, groups=16, seed=9)
            data = []
            for _ in range(4):
                A.sweep(S, 20)
                data.append(P.gather(S))
            P.train(torch.cat(data), steps=300, batch=2048, lr=2e-3)
        Es, Ms = [], []
        for r in range(ROUNDS):
            if P is not None:
                P.round(S, beta, seed=5, rnd=r, accepted=acc)
            A.sweep(S, 1)
            E, M = A.observables(S)
            Es.append(E.clone())
            Ms.append(M.abs().reshape(R).clone())
        Es = torch.stack(Es).cpu().numpy() / L ** 3
        Ms = torch.stack(Ms).cpu().numpy() / L ** 3
        res[arm] = []
        for series in (Es, Ms):
            tau = stats.integrated_tau(series)
            mean = series.mean()
            err = series.std() * np.sqrt(2 * tau / series.size)
            res[arm].append((mean, err))
        if P is not None:
            res["acceptance"] = acc.sum().item() / (ROUNDS * R * (L // 4) ** 3)
    for k in range(2):
        (m1, e1), (m2, e2) = res["plain"][k], res["learned"][k]
        assert abs(m1 - m2) < 2 * np.hypot(e1, e2), (k, res)
    assert res["acceptance"] > 0.0


def test_trained_network_decorrelates_faster_than_untrained():
    """What training gains. On a 32^3 lattice at T = 4.5115, block rounds (one colour step per block colour,
    then one plain sweep) with a network trained on the plain chain's blocks against the same rounds with the
    untrained network: the trained proposals are accepted for about half of all blocks (the untrained ones
    almost never), and the chain decorrelates faster: smaller tau_int of E and of |M| (Sokal window over 64
    chains of 3000 rounds). The gain is modest at these sizes: the block moves leave the long-wavelength modes
    to the plain sweeps."""
    _need_gpu()
    from spin_colour_kernel_b200 import stats
    from spin_colour_kernel_b200 import system as sy
    from spin_colour_kernel_b200.learned import BlockProposal
    from spin_colour_kernel_b200.sampler import Sampler
    L, R, T, K = 32, 64, 4.5115, 3000
    s = sy.ising("sc", L)
    A = Sampler(s, R, device="cuda", seed=31, packed=False)
    A.set_temperature(torch.full((R,), T))
    S = A.init_spins(seed=4)
    A.sweep(S, 1000)
    beta = torch.full((R,), 1.0 / T, dtype=torch.float32, device="cuda")
    trained = BlockProposal(L, R, groups=16, seed=9)
    data = []
    for _ in range(8):
        A.sweep(S, 25)
        data.append(trained.gather(S))
    trained.train(torch.cat(data), steps=800, batch=4096, lr=2e-3)
    untrained = BlockProposal(L, R, groups=16, seed=9)
    out = {}
    for name, P in (("trained", trained), ("untrained", untrained)):
        X = S.clone()
        acc = torch.zeros(R, dtype=torch.int32, device="cuda")
        Ms = torch.empty((K, R), dtype=torch.float64, device="cuda")
        Es = torch.empty((K, R), dtype=torch.float64, device="cuda")
        for r in range(K):
            P.round(X, beta, seed=13, rnd=r, accepted=acc)
            A.sweep(X, 1)
            E, M = A.observables(X)
            Ms[r].copy_(M.reshape(R).abs())
            Es[r].copy_(E)
        out[name] = {"tau_M": stats.integrated_tau(Ms.cpu().numpy() / L ** 3),
                     "tau_E": stats.integrated_tau(Es.cpu().numpy() / L ** 3),
                     "acceptance": acc.sum().item() / (K * R * (L // 4) ** 3)}
    t_, u_ = out["trained"], out["untrained"]
    assert t_["acceptance"] > 0.3 and t_["acceptance"] > 50 * u_["acceptance"], out
    assert t_["tau_E"] < 0.95 * u_["tau_E"] and t_["tau_M"] < u_["tau_M"], out
