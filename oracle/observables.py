"""FP64 observables restated in NumPy (oracle; test infrastructure only).

Follows Spin_Colour_Kernel/sampler.py:296-345: the bond part of the local field v_i = sum_bonds M_b s_j with
M_b = J_shell I + extra_b (neighbours outside an open box contribute nothing), the energy per replica
E = -1/2 sum_i s_i . v_i - sum_i h . s_i + sum_i [k1_i ((sx sy)^2 + (sx sz)^2 + (sy sz)^2) + k2 (sx sy sz)^2],
and the per-sublattice magnetization M[r, alpha, k] = sum over the sublattice of s_k.
"""

from __future__ import annotations

import numpy as np


def local_field(sys_, S: np.ndarray) -> np.ndarray:
    """S: (B, n, b, L3, L2, L1) spins (any dtype). Returns the float64 bond field, same shape."""
    D = sys_.crystal.D
    S64 = np.asarray(S, np.float64)
    v = np.zeros_like(S64)
    axis = {0: 5, 1: 4, 2: 3}
    for i, bd in enumerate(sys_.crystal.bonds):
        M = np.asarray(sys_.bond_matrix(i), np.float64)
        if not M.any():
            continue
        src = S64[:, :, bd.alpha2]
        valid = np.ones(sys_.shape[1:], np.float64)
        for k in range(D):
            d = bd.delta[k]
            if d == 0:
                continue
            src = np.roll(src, shift=-d, axis=axis[k] - 1)
            if not sys_.periodic[k]:
                Lk = sys_.box[k]
                idx = np.arange(Lk)
                ok = ((idx + d) >= 0) & ((idx + d) < Lk)
                shp = [1, 1, 1]
                shp[2 - k] = Lk
                valid = valid * ok.reshape(shp)
        v[:, :, bd.alpha] += np.einsum("kl,blzyx->bkzyx", M, src * valid)
    return v


def energy(sys_, S: np.ndarray) -> np.ndarray:
    S64 = np.asarray(S, np.float64)
    v = local_field(sys_, S64)
    E = -0.5 * (S64 * v).sum(axis=(1, 2, 3, 4, 5))
    if sys_.h is not None:
        E = E - (S64 * np.asarray(sys_.h, np.float64).reshape(1, -1, 1, 1, 1, 1)).sum(axis=(1, 2, 3, 4, 5))
    if sys_.cubic_k1 is not None:
        x, y, z = S64[:, 0], S64[:, 1], S64[:, 2]
        k1 = np.asarray(sys_.cubic_k1, np.float32).astype(np.float64)
        a = k1 * ((x * y) ** 2 + (x * z) ** 2 + (y * z) ** 2) + float(sys_.cubic_k2) * (x * y * z) ** 2
        E = E + a.sum(axis=(1, 2, 3, 4))
    return E


def magnetization(S: np.ndarray) -> np.ndarray:
    """(B, b, n) float64."""
    return np.asarray(S, np.float64).sum(axis=(3, 4, 5)).transpose(0, 2, 1)


def berg_luscher_q(layer: np.ndarray, valid: np.ndarray) -> np.ndarray:
    """Topological charge per replica of one layer (B, 3, Ny, Nx), FP64: every valid plaquette (Ny-1, Nx-1) cut
    into the spherical triangles (s00, s10, s11), (s00, s11, s01) of solid angle
    2 atan2(a . (b x c), 1 + a . b + b . c + c . a), summed and divided by 4 pi (anneal.py:69-80)."""
    s = np.moveaxis(np.asarray(layer, np.float64), 1, -1)
    s00, s10, s01, s11 = s[:, :-1, :-1], s[:, :-1, 1:], s[:, 1:, :-1], s[:, 1:, 1:]

    def omega(a, b, c):
        num = (a * np.cross(b, c)).sum(-1)
        den = 1.0 + (a * b).sum(-1) + (b * c).sum(-1) + (c * a).sum(-1)
        return 2.0 * np.arctan2(num, den)
    return ((omega(s00, s10, s11) + omega(s00, s11, s01)) * valid).sum(axis=(1, 2)) / (4.0 * np.pi)
