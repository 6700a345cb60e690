"""FP64 restatement of the learned block proposal (oracle; test infrastructure only).

The proposal has no counterpart in the reference; this file defines its mathematics for the checks of the GPU
kernels (forward, log-density, gradients, block geometry, proposal sampling, Metropolis-Hastings round):

  blocks    a cubic lattice (simple cubic Ising, periodic, L a multiple of 4) is cut into 4x4x4 blocks; block
            (bx, by, bz) has colour (bx & 1) | (by & 1) << 1 | (bz & 1) << 2, so two blocks of one colour share
            no bond and neither touches the other's boundary; a colour step updates all its blocks at once;
  inputs    the 96 boundary spins (faces -x, +x, -y, +y, -z, +z, 16 each, raster over the two other local
            coordinates, lower axis fastest) then the 64 block spins in autoregressive order `ORDER` (even
            sites of the block first, then odd sites, each sublattice (x%2, y%2, z%2) in raster order);
  network   masked autoregressive MLP (MADE, Germain et al. 2015): inputs -> H -> H -> H -> 64 logits, ReLU;
            spins are autoregressive over G groups of 64 / G consecutive positions (G = 64: one spin per step;
            G = 16: four spins of one half-sublattice per step, which share no bond); degrees: boundary 0,
            position p: p // S + 1 (S = 64 / G), hidden unit k: m_k = k G // H; masks: input i -> unit k iff
            deg(i) <= m_k, unit k -> unit k' iff m_k <= m_k', unit k -> logit p iff m_k <= p // S;
  density   log q(x | b) = sum_p log sigmoid(x_p * logit_p(x_<group(p), b)), x_p in {-1, +1};
  sampling  group by group: x_p = +1 iff u_p < sigmoid(logit_p), u_p uniform;
  MH        accept x' with min(1, exp(-beta (E(x') - E(x))) q(x | b) / q(x' | b)): u_acc < that ratio;
  loss      mean over a batch of -log q.

Random numbers of a colour step come from Philox4x32-10 (`philox.py`) with key
made_key(seed, round, colour) = (seed * 1000003 + (8 round + colour) * 7919 + 24680) mod 2147483629 and counter
17 uid + w, uid = replica * n_blocks + block (block raster bx + nb by + nb^2 bz): call w < 16 gives the uniforms
of positions 4w..4w+3, call 16 output 0 the acceptance uniform.

`bf16` rounds an array to bfloat16 (round to nearest even) and back, so the oracle can mirror the kernels'
storage precision (weights and activations in bfloat16, accumulation in float32 or wider).
"""

from __future__ import annotations

import numpy as np

from . import philox as PH

BS = 4                     # block edge
NS = BS ** 3               # spins per block
NB = 6 * BS * BS           # boundary spins per block
NCOL = 8


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (nearest, ties to even) and return them as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


# ------------------------------------------------------------------ block geometry
def _order() -> np.ndarray:
    subs = [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)]
    out = []
    for sx, sy, sz in subs:
        for lz in range(sz, BS, 2):
            for ly in range(sy, BS, 2):
                for lx in range(sx, BS, 2):
                    out.append(lx + BS * ly + BS * BS * lz)
    return np.array(out, np.int64)


ORDER = _order()                      # position p -> raster index t = lx + 4 ly + 16 lz
POS = np.argsort(ORDER)               # raster index -> position


def boundary_offsets() -> np.ndarray:
    """(96, 3) local coordinates (lx, ly, lz) of the boundary spins, in input order."""
    out = []
    for axis in range(3):
        for side in (-1, BS):
            others = [a for a in range(3) if a != axis]
            for b in range(BS):
                for a in range(BS):
                    c = [0, 0, 0]
                    c[axis] = side
                    c[others[0]] = a
                    c[others[1]] = b
                    out.append(c)
    return np.array(out, np.int64)


def face_pairs() -> np.ndarray:
    """(96, 2): (position of the block spin, boundary index) for every bond crossing the block surface."""
    bo = boundary_offsets()
    out = []
    for q, c in enumerate(bo):
        c = c.copy()
        c = np.clip(c, 0, BS - 1)
        t = c[0] + BS * c[1] + BS * BS * c[2]
        out.append((POS[t], q))
    return np.array(out, np.int64)


def internal_pairs() -> np.ndarray:
    """(144, 2) positions of the bonds inside a block."""
    out = []
    for lz in range(BS):
        for ly in range(BS):
            for lx in range(BS):
                t = lx + BS * ly + BS * BS * lz
                for d in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
                    x2, y2, z2 = lx + d[0], ly + d[1], lz + d[2]
                    if max(x2, y2, z2) < BS:
                        out.append((POS[t], POS[x2 + BS * y2 + BS * BS * z2]))
    return np.array(out, np.int64)


def block_origin(L: int, block: int):
    nb = L // BS
    return (block % nb) * BS, (block // nb % nb) * BS, (block // (nb * nb)) * BS


def blocks_of_colour(L: int, colour: int) -> np.ndarray:
    nb = L // BS
    b = np.arange(nb ** 3)
    bx, by, bz = b % nb, b // nb % nb, b // (nb * nb)
    return b[((bx & 1) | (by & 1) << 1 | (bz & 1) << 2) == colour]


def gather(spins: np.ndarray, blocks: np.ndarray):
    """spins (R, L, L, L) as [z, y, x] -> boundary (R, nblk, 96) and block spins (R, nblk, 64) in input order."""
    R, L = spins.shape[0], spins.shape[-1]
    bo = boundary_offsets()
    bnd = np.empty((R, len(blocks), NB), np.float64)
    blk = np.empty((R, len(blocks), NS), np.float64)
    for i, b in enumerate(blocks):
        x0, y0, z0 = block_origin(L, int(b))
        xs = (x0 + bo[:, 0]) % L
        ys = (y0 + bo[:, 1]) % L
        zs = (z0 + bo[:, 2]) % L
        bnd[:, i] = spins[:, zs, ys, xs]
        t = ORDER
        blk[:, i] = spins[:, z0 + t // 16, y0 + t // 4 % 4, x0 + t % 4]
    return bnd, blk


def scatter(spins: np.ndarray, blocks: np.ndarray, blk: np.ndarray, where: np.ndarray) -> None:
    """Write block spins (R, nblk, 64; input order) back where `where` (R, nblk) is true."""
    L = spins.shape[-1]
    t = ORDER
    for i, b in enumerate(blocks):
        x0, y0, z0 = block_origin(L, int(b))
        for r in np.nonzero(where[:, i])[0]:
            spins[r, z0 + t // 16, y0 + t // 4 % 4, x0 + t % 4] = blk[r, i]


# ------------------------------------------------------------------ network
def masks(n_boundary: int, n_spins: int, hidden: int, layers: int = 3, groups: int | None = None):
    G = n_spins if groups is None else groups
    S = n_spins // G
    grp = np.arange(n_spins) // S
    deg_in = np.concatenate([np.zeros(n_boundary, np.int64), grp + 1])
    m = np.arange(hidden) * G // hidden
    out = [(deg_in[None, :] <= m[:, None]).astype(np.float64)]
    for _ in range(layers - 1):
        out.append((m[None, :] <= m[:, None]).astype(np.float64))
    out.append((m[None, :] <= grp[:, None]).astype(np.float64))
    return out


def init_params(n_boundary: int, n_spins: int, hidden: int, layers: int = 3, seed: int = 0):
    """[(W, b)] in float32, Kaiming-uniform weights, zero biases."""
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


def sample(params, mk, boundary: np.ndarray, u: np.ndarray, groups: int, round_bf16: bool = True):
    """Autoregressive draw, group by group: x_p = +1 iff u_p < sigmoid(logit_p). Returns (x, logits of x)."""
    n, ns = u.shape
    S = ns // groups
    x = np.zeros((n, ns))
    for g in range(groups):
        logits, _ = forward(params, mk, boundary, x, round_bf16)
        sl = slice(g * S, (g + 1) * S)
        x[:, sl] = np.where(u[:, sl] < 1.0 / (1.0 + np.exp(-logits[:, sl])), 1.0, -1.0)
    logits, _ = forward(params, mk, boundary, x, round_bf16)
    return x, logits


def block_energy(spins: np.ndarray, boundary: np.ndarray, internal_pairs: np.ndarray, face_pairs: np.ndarray,
                 J: float = 1.0, h: float = 0.0) -> np.ndarray:
    """E of each block: -J (sum over internal bonds + sum over block-boundary bonds) - h sum of spins."""
    e = -(spins[:, internal_pairs[:, 0]] * spins[:, internal_pairs[:, 1]]).sum(axis=1)
    e -= (spins[:, face_pairs[:, 0]] * boundary[:, face_pairs[:, 1]]).sum(axis=1)
    return J * e - h * spins.sum(axis=1)


def mh_log_ratio(beta, e_old, e_new, logq_old, logq_new):
    """log of exp(-beta (E' - E)) q(x | b) / q(x' | b)."""
    return -beta * (e_new - e_old) + logq_old - logq_new


# ------------------------------------------------------------------ one colour step
def made_key(seed: int, rnd: int, colour: int) -> int:
    v = int(seed) * 1000003 + (8 * int(rnd) + int(colour)) * 7919 + 24680
    r = abs(v) % 2147483629
    return r if v >= 0 else -r


def step_uniforms(seed: int, rnd: int, colour: int, uids: np.ndarray):
    """(uniforms of the 64 positions (N, 64), acceptance uniform (N,)) of blocks with global ids `uids`."""
    key = made_key(seed, rnd, colour)
    uids = np.asarray(uids, np.int64)
    u = np.empty((len(uids), NS), np.float32)
    for w in range(NS // 4):
        u4 = PH.uniform4(key, PH.int32_counter(uids * 17 + w))
        u[:, 4 * w:4 * w + 4] = u4.T
    acc = PH.uniform4(key, PH.int32_counter(uids * 17 + 16))[0]
    return u, acc


def colour_step(spins: np.ndarray, params, mk, beta: np.ndarray, seed: int, rnd: int, colour: int, groups: int,
                J: float = 1.0):
    """One colour step on int spins (R, L, L, L) in place. Returns a dict of per-block quantities."""
    R, L = spins.shape[0], spins.shape[-1]
    blocks = blocks_of_colour(L, colour)
    nbt = (L // BS) ** 3
    bnd, cur = gather(spins, blocks)
    uids = (np.arange(R)[:, None] * nbt + blocks[None, :]).reshape(-1)
    u, acc = step_uniforms(seed, rnd, colour, uids)
    b2 = bnd.reshape(-1, NB)
    x = cur.reshape(-1, NS)
    xp, lp = sample(params, mk, b2, u.astype(np.float64), groups)
    lx, _ = forward(params, mk, b2, x)
    lq_new, lq_old = log_density(lp, xp), log_density(lx, x)
    ip, fp = internal_pairs(), face_pairs()
    dE = block_energy(xp, b2, ip, fp, J) - block_energy(x, b2, ip, fp, J)
    bet = np.repeat(np.asarray(beta, np.float64), len(blocks))
    logr = mh_log_ratio(bet, 0.0, dE, lq_old, lq_new)
    accept = acc.astype(np.float64) < np.exp(np.minimum(logr, 0.0))
    scatter(spins, blocks, xp.reshape(R, len(blocks), NS), accept.reshape(R, len(blocks)))
    return {"x_new": xp, "x_old": x, "u": u, "u_acc": acc, "logq_new": lq_new, "logq_old": lq_old, "dE": dE,
            "logr": logr, "accept": accept, "logits_new": lp, "logits_old": lx, "blocks": blocks}
