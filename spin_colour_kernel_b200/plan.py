"""Host side of the boundary: the C descriptor of a System and the host-built acceptance tables.

`describe(system)` lowers a System to the sck_system_desc of include/sck.h. The bonds of each sublattice are
listed in local-field accumulation order: bonds grouped by their float J in order of first appearance over
the bond table, members in table order, groups with J = 0 and no extra matrix left out; extra matrices take
slots in bond-table order (Spin_Colour_Kernel/generator.py:215-273). Classes are colour-major, then
sublattice, skipping classes without an active site (sampler.py:128-129).

`ising_table` builds the per-replica acceptance table of Ising chains. An Ising energy change is fixed by the
own spin, the integer neighbour sum G_g of every applied coupling group and the neighbour of every bond with
a non-zero extra coupling; the table holds, for every such key, exp(-beta dE) (Metropolis) or exp(beta dE)
(Barker) evaluated with the float32 operations of the generated kernel (v = sum_g J_g G_g, + E n, + h;
dE = -((t - s) v), t = -s) and NumPy's float32 exp — the functions the reference's CPU path evaluates.
Key layout (shared with the kernels): key = [s > 0] + sum_g (G_g + z_g) stride_g + sum_e (n_e + 1) stride_e
with mixed-radix strides 2, 2 (2 z_0 + 1), ... over applied groups, then extra slots.

`p_table` / `p_fixed` are the bitwise acceptance tables of bitwise.py:79-110.
"""

from __future__ import annotations

import numpy as np

from . import _lib as L


def coupling_groups(sys_, a: int):
    """[(J (float), [bond indices])] of sublattice a in first-appearance order, and its extra bonds."""
    groups: dict[float, list[int]] = {}
    extras: list[int] = []
    for i, bd in enumerate(sys_.crystal.bonds):
        if bd.alpha != a:
            continue
        groups.setdefault(float(sys_.J.get(bd.shell, 0.0)), []).append(i)
        if i in sys_.extra:
            extras.append(i)
    kept = [(J, m) for J, m in groups.items() if J != 0.0 or any(i in sys_.extra for i in m)]
    return kept, extras


def sweep_classes(sys_) -> list[tuple[int, int]]:
    cm, m = sys_.colour_map(), sys_.site_mask()
    return [(c, a) for c in range(sys_.colouring.n_colours) for a in range(sys_.b) if np.any((cm[a] == c) & m[a])]


def describe(sys_) -> L.SystemDesc:
    d = L.SystemDesc()
    d.abi_version = L.ABI_VERSION
    d.n, d.dim, d.b = sys_.n, sys_.crystal.D, sys_.b
    for k, v in enumerate((sys_.L1, sys_.L2, sys_.L3)):
        d.L[k] = v
    per = list(sys_.periodic) + [False] * (3 - sys_.crystal.D)
    for k in range(3):
        d.periodic[k] = int(bool(per[k]))
    d.acceptance = L.BARKER if sys_.acceptance == "barker" else L.METROPOLIS
    d.has_mask = int(sys_.mask is not None)
    d.has_cubic = int(sys_.cubic_k1 is not None)
    if sys_.h is not None:
        for k in range(sys_.n):
            d.h[k] = float(np.float32(sys_.h[k]))
            d.h64[k] = float(sys_.h[k])
    d.k2 = float(np.float32(sys_.cubic_k2))
    d.k2_64 = float(sys_.cubic_k2)
    col = sys_.colouring
    if len(col.m) > L.MAX_FACTORS:
        raise ValueError("colouring has more cyclic factors than the kernels support")
    d.n_factors = len(col.m)
    for r, mr in enumerate(col.m):
        d.m[r] = mr
        for k in range(sys_.crystal.D):
            d.K[r][k] = int(col.K[r][k]) % mr
        for a in range(sys_.b):
            d.o[a][r] = int(col.o[a][r]) % mr
    classes = sweep_classes(sys_)
    if len(classes) > L.MAX_CLASSES:
        raise ValueError("too many colour classes for the kernels")
    d.n_classes = len(classes)
    for i, (c, a) in enumerate(classes):
        d.classes[i][0], d.classes[i][1] = c, a
    bonds = sys_.crystal.bonds
    for a in range(sys_.b):
        groups, extras = coupling_groups(sys_, a)
        sub = d.sub[a]
        if len(groups) > L.MAX_GROUPS or len(extras) > L.MAX_EXTRA:
            raise ValueError("too many coupling groups or extra matrices on one sublattice")
        nb = 0
        for g, (J, members) in enumerate(groups):
            for i in members:
                if nb >= L.MAX_BONDS:
                    raise ValueError(f"more than {L.MAX_BONDS} bonds leave one sublattice")
                bd = bonds[i]
                e = sub.bonds[nb]
                e.alpha2 = bd.alpha2
                delta = list(bd.delta) + [0] * (3 - sys_.crystal.D)
                for k in range(3):
                    e.d[k] = int(delta[k])
                e.group = g
                e.extra = extras.index(i) if i in sys_.extra else -1
                e.J64 = float(sys_.J.get(bd.shell, 0.0))
                nb += 1
            sub.group_end[g] = nb
            sub.group_J[g] = float(np.float32(J))
            sub.group_apply[g] = int(J != 0.0)
        sub.n_bonds, sub.n_groups, sub.n_extra = nb, len(groups), len(extras)
        for s, i in enumerate(extras):
            E = np.asarray(sys_.extra[i], np.float64)
            for k in range(sys_.n):
                for l in range(sys_.n):
                    sub.extra[s][3 * k + l] = float(np.float32(E[k, l]))
                    sub.extra64[s][3 * k + l] = float(E[k, l])
    return d


# ----------------------------------------------------------------------------------------------- Ising table
def ising_key_layout(sys_, a: int):
    """[(J float32, z_g)] of applied groups and [E float32] of extra slots that enter the key, in key order."""
    groups, extras = coupling_groups(sys_, a)
    applied = [(np.float32(J), len(m)) for J, m in groups if J != 0.0]
    slots = [np.float32(np.asarray(sys_.extra[i])[0, 0]) for i in extras if np.asarray(sys_.extra[i])[0, 0] != 0.0]
    return applied, slots


def ising_keys(sys_, a: int) -> int:
    applied, slots = ising_key_layout(sys_, a)
    return int(2 * np.prod([2 * z + 1 for _, z in applied], dtype=np.int64) * 3 ** len(slots))


def ising_table(sys_, beta: np.ndarray, keys: int) -> np.ndarray:
    """float32 [len(beta), b, keys] acceptance table (see module docstring)."""
    beta = np.asarray(beta, np.float32).reshape(-1)
    out = np.zeros((beta.size, sys_.b, keys), np.float32)
    h0 = np.float32(sys_.h[0]) if (sys_.h is not None and sys_.h[0] != 0.0) else None
    for a in range(sys_.b):
        applied, slots = ising_key_layout(sys_, a)
        ka = ising_keys(sys_, a)
        k = np.arange(ka, dtype=np.int64)
        s = np.where(k % 2 == 1, np.float32(1.0), np.float32(-1.0)).astype(np.float32)
        rest = k // 2
        v = np.zeros(ka, np.float32)
        for J, z in applied:
            G = (rest % (2 * z + 1) - z).astype(np.float32)
            rest = rest // (2 * z + 1)
            v = v + J * G
        for E in slots:
            n = (rest % 3 - 1).astype(np.float32)
            rest = rest // 3
            v = v + E * n
        if h0 is not None:
            v = v + h0
        t = -s
        dE = -((t - s) * v)
        with np.errstate(over="ignore"):
            if sys_.acceptance == "barker":
                e = np.exp(beta[:, None] * dE[None, :])
            else:
                e = np.exp((-beta)[:, None] * dE[None, :])
        out[:, a, :ka] = e
    return out


# ---------------------------------------------------------------------------------------------- bitwise
def bitwise_check(sys_):
    """(J, h, Z) of a system the bitwise kernels accept; ValueError otherwise (bitwise.py:59-71)."""
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


def _p64(sys_, beta) -> np.ndarray:
    J, h, Z = bitwise_check(sys_)
    beta = np.asarray(beta, np.float64).reshape(-1)
    p = np.zeros((beta.size, 2, Z + 1, Z + 1), np.float64)
    for s in (0, 1):
        for ze in range(Z + 1):
            k = np.arange(ze + 1)
            x = beta[:, None] * (2.0 * J * (ze - 2 * k) + 2.0 * h * (2 * s - 1))[None, :]
            if sys_.acceptance == "barker":
                p[:, s, ze, : ze + 1] = 0.5 * (1.0 - np.tanh(0.5 * x))
            else:
                p[:, s, ze, : ze + 1] = np.exp(-np.maximum(x, 0.0))
    return p


def p_table(sys_, beta) -> np.ndarray:
    """Shared mode: float32 p[word, s, z_eff, k]."""
    return _p64(sys_, beta).astype(np.float32)


def p_fixed(sys_, beta) -> np.ndarray:
    """Independent mode: int64 P = floor(p 2^32) in [0, 2^32]."""
    return np.clip(np.floor(_p64(sys_, beta) * 2.0 ** 32).astype(np.int64), 0, 2 ** 32)
