"""The colour-class sweep restated in NumPy float32 (oracle; test infrastructure only).

One class launch of the reference's generated kernel (Spin_Colour_Kernel/generator.py:150-319) updates every
site of one (colour, sublattice) class of every replica. Here that launch is one vectorised NumPy step over
all sites of the class and all replicas, with the kernel's float32 operations in the kernel's order. The
reference's CPU path (the Triton interpreter) evaluates the same operations with the same NumPy functions
(np.exp, np.cos, np.sin, np.sqrt on float32 arrays), so this restatement reproduces it bit for bit; the
golden fixtures pin that.

Arithmetic of one attempt at site i of replica r (generator.py line numbers):
  local field :215-273  per sublattice, bonds grouped by their float J in first-appearance order; per group
                        g_k = sum of neighbour components (0 outside an open box), v_k += J * g_k; then
                        v_k += sum_l E_kl n_l for each bond with an extra matrix E; then v_k += h_k
  proposal    :275-289  (u0, u1, u2, u3) = rand4x(key, int32(r * nsite + i)); Ising t = -s;
                        XY phi = f32(2 pi) u1, t = (cos phi, sin phi); Heisenberg cz = 2 u1 - 1,
                        phi = f32(2 pi) u2, rr = sqrt(max(1 - cz^2, 0)), t = (rr cos phi, rr sin phi, cz)
  energy      :291-299  dE = -sum_k (t_k - s_k) v_k, plus cubic anisotropy a(t) - a(s) with
                        a(p) = k1 ((p0 p1)^2 + (p0 p2)^2 + (p1 p2)^2) + k2 (p0 p1 p2)^2
  acceptance  :300-305  Metropolis u0 < exp(-beta dE); Barker u0 (1 + exp(beta dE)) < 1
  store       :306-318  where(accepted, t, s), cast to the storage type, on updated sites only
"""

from __future__ import annotations

import numpy as np

from . import philox

F32 = np.float32
TWO_PI_F32 = np.float32(6.283185307179586)


def classes(sys_) -> list[tuple[int, int]]:
    """Sweep order: colour-major, then sublattice; classes without an active site are skipped."""
    cm, m = sys_.colour_map(), sys_.site_mask()
    return [(c, a) for c in range(sys_.colouring.n_colours) for a in range(sys_.b) if np.any((cm[a] == c) & m[a])]


def field_groups(sys_, a: int):
    """Bonds of sublattice a grouped by float J (dict order = first appearance) and the bonds with extras."""
    groups: dict[float, list[int]] = {}
    extras: list[int] = []
    for i, bd in enumerate(sys_.crystal.bonds):
        if bd.alpha != a:
            continue
        groups.setdefault(float(sys_.J.get(bd.shell, 0.0)), []).append(i)
        if i in sys_.extra:
            extras.append(i)
    return groups, extras


def neighbour(sys_, bd, z, y, x):
    """Neighbour coordinates of sites (z, y, x) along bond bd and their validity (open boundaries)."""
    D = sys_.crystal.D
    d = list(bd.delta) + [0] * (3 - D)
    per = list(sys_.periodic) + [False] * (3 - D)
    L = (sys_.L1, sys_.L2, sys_.L3)
    out, ok = [], np.ones(x.shape, bool)
    for k, c in enumerate((x, y, z)):
        q = c + d[k]
        if d[k] != 0:
            if per[k]:
                q = (c + d[k] % L[k]) % L[k]
            else:
                ok &= (q >= 0) & (q < L[k])
                q = np.where(ok, q, 0)
        out.append(q)
    return out[2], out[1], out[0], ok


def class_update(sys_, S: np.ndarray, dst: np.ndarray, beta: np.ndarray, base_seed: int, sweep: int,
                 colour: int, alpha: int, reps=None) -> None:
    """One class launch. S, dst: (B, n, b, L3, L2, L1) storage arrays (dst may be S). colour < 0 is the
    synchronous control: every site of the sublattice, read from S, written to dst. `reps` gives the global
    replica index of each row of S (default 0 .. B-1): it enters the Philox counter, so a few replicas of a
    large batch can be checked on their own."""
    n = sys_.n
    B = S.shape[0]
    reps = np.arange(B, dtype=np.int64) if reps is None else np.asarray(reps, np.int64)
    b, L3, L2, L1 = sys_.shape
    nsite = b * L3 * L2 * L1
    mask = sys_.site_mask()
    sel = mask[alpha] if colour < 0 else (sys_.colour_map()[alpha] == colour) & mask[alpha]
    z, y, x = np.nonzero(sel)
    if z.size == 0:
        return
    own = alpha * L3 * L2 * L1 + z * L2 * L1 + y * L1 + x
    s = [S[:, k, alpha, z, y, x].astype(F32) for k in range(n)]            # (B, ns) each
    v = [np.zeros((B, z.size), F32) for _ in range(n)]
    groups, extras = field_groups(sys_, alpha)
    saved: dict[int, list[np.ndarray]] = {}
    bonds = sys_.crystal.bonds
    for Jv, members in groups.items():
        if Jv == 0.0 and not any(i in sys_.extra for i in members):
            continue
        g = [np.zeros((B, z.size), F32) for _ in range(n)]
        for i in members:
            zq, yq, xq, ok = neighbour(sys_, bonds[i], z, y, x)
            a2 = bonds[i].alpha2
            t = [np.where(ok[None, :], S[:, k, a2, zq, yq, xq].astype(F32), F32(0.0)) for k in range(n)]
            for k in range(n):
                g[k] = g[k] + t[k]
            if i in sys_.extra:
                saved[i] = t
        if Jv != 0.0:
            for k in range(n):
                v[k] = v[k] + F32(Jv) * g[k]
    for i in extras:
        E = sys_.extra[i]
        for k in range(n):
            terms = [F32(E[k, l]) * saved[i][l] for l in range(n) if E[k, l] != 0.0]
            if terms:
                tot = terms[0]
                for tm in terms[1:]:
                    tot = tot + tm
                v[k] = v[k] + tot
    if sys_.h is not None:
        for k in range(n):
            if sys_.h[k] != 0.0:
                v[k] = v[k] + F32(sys_.h[k])
    key = philox.sweep_seed(base_seed, sweep)
    key = int(np.int64(key).astype(np.int32))
    ctr = philox.int32_counter(reps[:, None] * nsite + own[None, :])
    u = philox.uniform4(key, ctr.reshape(-1)).reshape(4, B, z.size)
    u0, u1, u2 = u[0], u[1], u[2]
    with np.errstate(over="ignore", invalid="ignore"):
        if n == 1:
            t = [-s[0]]
        elif n == 2:
            phi = TWO_PI_F32 * u1
            t = [np.cos(phi), np.sin(phi)]
        else:
            cz = F32(2.0) * u1 - F32(1.0)
            phi = TWO_PI_F32 * u2
            rr = np.sqrt(np.maximum(F32(1.0) - cz * cz, F32(0.0)))
            t = [rr * np.cos(phi), rr * np.sin(phi), cz]
        acc_sum = (t[0] - s[0]) * v[0]
        for k in range(1, n):
            acc_sum = acc_sum + (t[k] - s[k]) * v[k]
        dE = -acc_sum
        if sys_.cubic_k1 is not None:
            k1 = np.asarray(sys_.cubic_k1, F32)[alpha, z, y, x][None, :]
            k2 = F32(sys_.cubic_k2)

            def aniso(p):
                q01, q02, q12 = p[0] * p[1], p[0] * p[2], p[1] * p[2]
                tri = p[0] * p[1] * p[2]
                return k1 * ((q01 * q01 + q02 * q02) + q12 * q12) + (k2 * tri) * tri
            dE = dE + (aniso(t) - aniso(s))
        bt = np.asarray(beta, F32).reshape(B, 1)
        if sys_.acceptance == "barker":
            acc = (u0 * (F32(1.0) + np.exp(bt * dE))) < F32(1.0)
        else:
            acc = u0 < np.exp((-bt) * dE)
    for k in range(n):
        dst[:, k, alpha, z, y, x] = np.where(acc, t[k], s[k]).astype(dst.dtype)


def sweep(sys_, S: np.ndarray, beta: np.ndarray, state: list[int], n: int = 1, reps=None) -> np.ndarray:
    """n sweeps in place; state = [base_seed, sweep] advances by one per sweep."""
    order = classes(sys_)
    for _ in range(n):
        for c, a in order:
            class_update(sys_, S, S, beta, state[0], state[1], c, a, reps)
        state[1] += 1
    return S


def sync_sweep(sys_, S: np.ndarray, beta: np.ndarray, state: list[int], n: int = 1) -> np.ndarray:
    """The negative control: every site updated from the previous state in one step."""
    for _ in range(n):
        dst = S.copy()
        for a in range(sys_.b):
            class_update(sys_, S, dst, beta, state[0], state[1], -1, a)
        S[...] = dst
        state[1] += 1
    return S
