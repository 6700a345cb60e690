"""Bitwise multi-spin-coded Ising restated on unpacked spins (oracle; test infrastructure only).

Follows Spin_Colour_Kernel/bitwise.py:59-246. Word w holds replicas 32 w .. 32 w + 31. For a site i with
present neighbours j (inside the box and the mask, bonds with J != 0), z_eff = number of present neighbours
and k = number of anti-aligned ones; replica r flips when its draw is below table[w, s, z_eff, k] (s = 1 for
spin +1 when the system has a field, else 0):
  shared mode      one float32 uniform per (word, site, sweep): output w % 4 of
                   rand4x(key, int32((w // 4) * nsite + i)), compared with the float32 table p (p_table);
  independent mode one 32-bit integer U per (replica, site, sweep): bit 31 - l of U of replica 32 w + j is bit
                   j of R_l, R_{4g+q} = output q of randint4x(key_g, int32(w * nsite + i)),
                   key_g = (key + (g + 1) * 104729) mod 2147483629; flip iff U < P (p_fixed, int64).
The tables are built in float64: dE = 2 J (z_eff - 2 k) + 2 h sigma, Metropolis exp(-max(beta dE, 0)),
Barker (1 - tanh(beta dE / 2)) / 2; p_table casts to float32, p_fixed takes floor(p 2^32) clipped to [0, 2^32].
"""

from __future__ import annotations

import numpy as np

from . import philox
from .sweep import classes, neighbour

WORD = 32
GROUP_KEY_STEP = 104729
LEVELS = 32


def check(sys_):
    """(J, h, Z) of a system the bitwise chain accepts; ValueError otherwise."""
    if sys_.n != 1:
        raise ValueError("bitwise multi-spin coding is for Ising (n = 1) only")
    if sys_.extra:
        raise ValueError("bitwise multi-spin coding needs isotropic exchange only (no extra bond matrices)")
    if sys_.cubic_k1 is not None:
        raise ValueError("bitwise multi-spin coding does not support anisotropy")
    Js = {float(sys_.J.get(bd.shell, 0.0)) for bd in sys_.crystal.bonds} - {0.0}
    if len(Js) != 1:
        raise ValueError(f"bitwise multi-spin coding needs one uniform coupling J on every bond, got {sorted(Js)}")
    h = float(sys_.h[0]) if sys_.h is not None else 0.0
    Z = max(sum(1 for bd in sys_.crystal.bonds if bd.alpha == a and sys_.J.get(bd.shell, 0.0) != 0.0)
            for a in range(sys_.b))
    return Js.pop(), h, Z


def p64(sys_, beta) -> np.ndarray:
    J, h, Z = check(sys_)
    beta = np.asarray(beta, np.float64).reshape(-1)
    p = np.zeros((beta.size, 2, Z + 1, Z + 1), np.float64)
    for s in (0, 1):
        sigma = 2 * s - 1
        for ze in range(Z + 1):
            k = np.arange(ze + 1)
            x = beta[:, None] * (2.0 * J * (ze - 2 * k) + 2.0 * h * sigma)[None, :]
            if sys_.acceptance == "barker":
                p[:, s, ze, : ze + 1] = 0.5 * (1.0 - np.tanh(0.5 * x))
            else:
                p[:, s, ze, : ze + 1] = np.exp(-np.maximum(x, 0.0))
    return p


def p_table(sys_, beta) -> np.ndarray:
    return p64(sys_, beta).astype(np.float32)


def p_fixed(sys_, beta) -> np.ndarray:
    return np.clip(np.floor(p64(sys_, beta) * 2.0 ** 32).astype(np.int64), 0, 2 ** 32)


def shared_uniforms(base_seed: int, sweep: int, n_words: int, nsite: int, words=None) -> np.ndarray:
    """Uniform of every (word, site) of one sweep, (n_words, nsite) float32; `words` = global word indices."""
    words = np.arange(n_words, dtype=np.int64) if words is None else np.asarray(words, np.int64)
    ctr = (words // 4)[:, None] * nsite + np.arange(nsite, dtype=np.int64)[None, :]
    u = philox.uniform4(philox.sweep_seed(base_seed, sweep), philox.int32_counter(ctr).reshape(-1))
    u = u.reshape(4, words.size, nsite)
    return u[words % 4, np.arange(words.size)]


def lane_integers(base_seed: int, sweep: int, n_words: int, nsite: int, words=None) -> np.ndarray:
    """The 32-bit integer U of every (replica, site) of one sweep, (32 n_words, nsite) int64."""
    words = np.arange(n_words, dtype=np.int64) if words is None else np.asarray(words, np.int64)
    n_words = words.size
    key = philox.sweep_seed(base_seed, sweep)
    ctr = philox.int32_counter(words[:, None] * nsite + np.arange(nsite, dtype=np.int64)[None, :]).reshape(-1)
    lane = np.arange(WORD, dtype=np.uint64)
    U = np.zeros((n_words, WORD, nsite), np.int64)
    for g in range(LEVELS // 4):
        kg = (key + (g + 1) * GROUP_KEY_STEP) % 2147483629
        R = philox.raw4(kg, ctr).astype(np.uint64).reshape(4, n_words, 1, nsite)
        for q in range(4):
            bit = ((R[q] >> lane[None, :, None]) & np.uint64(1)).astype(np.int64)
            U |= bit << (LEVELS - 1 - (4 * g + q))
    return U.reshape(n_words * WORD, nsite)


def sweep(sys_, spins: np.ndarray, table: np.ndarray, base_seed: int, sweep_idx: int,
          independent: bool = False, words=None) -> np.ndarray:
    """One sweep of every replica on unpacked spins (B, b, L3, L2, L1) of +-1 (0 on masked sites).

    `words` gives the global word index of each block of 32 rows (default 0, 1, ...), so the replicas of a few
    words of a large batch can be checked on their own; `table` is indexed by local word."""
    _, h, _ = check(sys_)
    S = np.array(spins, dtype=np.int64, copy=True)
    B = S.shape[0]
    b, L3, L2, L1 = sys_.shape
    nsite = b * L3 * L2 * L1
    W = -(-B // WORD)
    mask = sys_.site_mask()
    cm = sys_.colour_map()
    draws = (lane_integers(base_seed, sweep_idx, W, nsite, words)[:B] if independent
             else shared_uniforms(base_seed, sweep_idx, W, nsite, words))
    word = np.arange(B) // WORD
    for c, a in classes(sys_):
        z, y, x = np.nonzero((cm[a] == c) & mask[a])
        site = a * L3 * L2 * L1 + z * L2 * L1 + y * L1 + x
        ze = np.zeros(z.size, np.int64)
        tot = np.zeros((B, z.size), np.int64)
        for bd in sys_.crystal.bonds:
            if bd.alpha != a or sys_.J.get(bd.shell, 0.0) == 0.0:
                continue
            zq, yq, xq, ok = neighbour(sys_, bd, z, y, x)
            ok = ok & mask[bd.alpha2, zq, yq, xq]
            ze += ok
            tot += np.where(ok[None, :], S[:, bd.alpha2, zq, yq, xq], 0)
        si = S[:, a, z, y, x]
        kk = (ze[None, :] - si * tot) // 2
        s_idx = (si > 0).astype(np.int64) if h != 0.0 else np.zeros_like(si)
        p = table[word[:, None], s_idx, ze[None, :], kk]
        u = draws[:, site] if independent else draws[word[:, None], site[None, :]]
        S[:, a, z, y, x] = np.where(u < p, -si, si)
    return S.astype(spins.dtype)
