"""FP64 restatement of the learned block proposal (oracle; test infrastructure only).

The proposal has no counterpart in the reference; this file defines its mathematics for the checks of the GPU
kernels (forward, log-density, gradients, Metropolis-Hastings ratio):

  network   masked autoregressive MLP (MADE, Germain et al. 2015) over the B block spins in raster order,
            conditioned on the NB boundary spins: inputs (boundary, spins) -> H -> H -> H -> B logits, ReLU;
            degrees: boundary inputs 0, spin j: j + 1, hidden unit k: m_k = floor(k B / H) (sorted, so the
            inputs a unit may read are a prefix of the previous layer); masks: input i -> unit k iff
            deg(i) <= m_k, unit k -> unit k' iff m_k <= m_k', unit k -> logit j iff m_k <= j;
  density   log q(x | b) = sum_j log sigmoid(x_j * logit_j(x_<j, b)), x_j in {-1, +1};
  loss      mean over a batch of -log q;
  MH ratio  accept x' with min(1, exp(-beta (E(x') - E(x))) q(x | b) / q(x' | b)).

`bf16` rounds an array to bfloat16 (round to nearest even) and back, so the oracle can mirror the kernels'
storage precision (weights and activations in bfloat16, accumulation in float32 or wider).
"""

from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (nearest, ties to even) and return them as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def masks(n_boundary: int, n_spins: int, hidden: int, layers: int = 3):
    deg_in = np.concatenate([np.zeros(n_boundary, np.int64), np.arange(1, n_spins + 1)])
    m = np.arange(hidden) * n_spins // hidden
    out = [(deg_in[None, :] <= m[:, None]).astype(np.float64)]
    for _ in range(layers - 1):
        out.append((m[None, :] <= m[:, None]).astype(np.float64))
    out.append((m[None, :] <= np.arange(n_spins)[:, None]).astype(np.float64))
    return out


def init_params(n_boundary: int, n_spins: int, hidden: int, layers: int = 3, seed: int = 0):
    """[(W, b)] in float32, Kaiming-uniform weights scaled by the mask density, zero biases."""
    rng = np.random.default_rng(seed)
    sizes = [n_boundary + n_spins] + [hidden] * layers + [n_spins]
    params = []
    for fan_in, fan_out in zip(sizes[:-1], sizes[1:]):
        bound = np.sqrt(6.0 / fan_in)
        params.append((rng.uniform(-bound, bound, (fan_out, fan_in)).astype(np.float32),
                       np.zeros(fan_out, np.float32)))
    return params


def forward(params, mk, boundary: np.ndarray, spins: np.ndarray, round_bf16: bool = True):
    """Logits (batch, n_spins) and the layer inputs kept for the backward pass."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    x = r(np.concatenate([boundary, spins], axis=1))
    acts = [x]
    h = x
    for li, ((W, b), M) in enumerate(zip(params, mk)):
        z = h @ (r(W) * M).T + np.asarray(b, np.float64)
        if li < len(params) - 1:
            h = r(np.maximum(z, 0.0))
            acts.append(h)
        else:
            h = z
    return h, acts


def log_density(logits: np.ndarray, spins: np.ndarray) -> np.ndarray:
    t = spins * logits
    return -(np.logaddexp(0.0, -t)).sum(axis=1)


def loss_and_grads(params, mk, boundary, spins, round_bf16: bool = True):
    """Mean negative log-density and its gradients [(dW, db)] (dW already masked)."""
    logits, acts = forward(params, mk, boundary, spins, round_bf16)
    n = spins.shape[0]
    loss = -log_density(logits, spins).mean()
    # d(-log sigmoid(s t))/dt = -s sigmoid(-s t)
    g = -spins * (1.0 / (1.0 + np.exp(spins * logits))) / n
    grads = [None] * len(params)
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    for li in range(len(params) - 1, -1, -1):
        W, _ = params[li]
        Wm = r(W) * mk[li]
        grads[li] = ((g.T @ acts[li]) * mk[li], g.sum(axis=0))
        if li > 0:
            g = (g @ Wm) * (acts[li] > 0)
    return loss, grads


def block_energy(spins: np.ndarray, boundary: np.ndarray, internal_pairs: np.ndarray, face_pairs: np.ndarray,
                 J: float = 1.0, h: float = 0.0) -> np.ndarray:
    """E of each block: -J (sum over internal bonds + sum over block-boundary bonds) - h sum of spins."""
    e = -(spins[:, internal_pairs[:, 0]] * spins[:, internal_pairs[:, 1]]).sum(axis=1)
    e -= (spins[:, face_pairs[:, 0]] * boundary[:, face_pairs[:, 1]]).sum(axis=1)
    return J * e - h * spins.sum(axis=1)


def mh_log_ratio(beta, e_old, e_new, logq_old, logq_new):
    """log of exp(-beta (E' - E)) q(x | b) / q(x' | b)."""
    return -beta * (e_new - e_old) + logq_old - logq_new
