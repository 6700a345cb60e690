"""ctypes front end of oracle/cpu_sweep.c (oracle; test infrastructure and timed CPU baseline only).

Build recipe: `python -m oracle.native` (also run by __graft_entry__.build) compiles cpu_sweep.c with gcc,
OpenMP and -ffp-contract=off into oracle/_build/libsckoracle.so (git-ignored; it travels to the GPU box).
The descriptor is built here from the System with the oracle's own grouping rule (oracle/sweep.py).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import time
from pathlib import Path

import numpy as np

from .sweep import classes, field_groups

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_sweep.c"
LIB = HERE / "_build" / "libsckoracle.so"
_i32, _f32 = ctypes.c_int32, ctypes.c_float


class _Bond(ctypes.Structure):
    _fields_ = [("a2", _i32), ("dx", _i32), ("dy", _i32), ("dz", _i32), ("extra", _i32)]


class _Desc(ctypes.Structure):
    _fields_ = [("n", _i32), ("b", _i32), ("L", _i32 * 3), ("periodic", _i32 * 3), ("acceptance", _i32),
                ("h", _f32 * 3), ("has_cubic", _i32), ("k2", _f32), ("r", _i32), ("m", _i32 * 4),
                ("K", (_i32 * 3) * 4), ("o", (_i32 * 4) * 4), ("n_classes", _i32), ("classes", (_i32 * 2) * 128),
                ("n_bonds", _i32 * 4), ("n_groups", _i32 * 4), ("group_end", (_i32 * 8) * 4), ("J", (_f32 * 8) * 4),
                ("apply", (_i32 * 8) * 4), ("n_extra", _i32 * 4), ("E", ((_f32 * 9) * 8) * 4),
                ("bonds", (_Bond * 64) * 4)]


_lib = None


def build(force: bool = False) -> Path:
    LIB.parent.mkdir(exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", str(SRC),
               "-o", str(LIB), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB


def available() -> bool:
    try:
        _load()
        return True
    except OSError:
        return False


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise OSError("oracle C port not built")
        L = ctypes.CDLL(str(LIB))
        L.oracle_sweep.argtypes = [ctypes.POINTER(_Desc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, _i32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, _i32, _i32,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_sweep.restype = _i32
        L.oracle_bitwise_sweep.argtypes = [ctypes.POINTER(_Desc), ctypes.c_void_p, ctypes.c_void_p, _i32,
                                           ctypes.c_void_p, ctypes.c_void_p, _i32, _i32, _i32, ctypes.c_int64,
                                           ctypes.c_int64, _i32, _i32]
        L.oracle_bitwise_sweep.restype = _i32
        L.oracle_max_threads.restype = _i32
        L.oracle_desc_size.restype = _i32
        if L.oracle_desc_size() != ctypes.sizeof(_Desc):
            raise OSError("oracle descriptor layout mismatch")
        _lib = L
    return _lib


def threads() -> int:
    return int(_load().oracle_max_threads())


def describe(sys_) -> _Desc:
    d = _Desc()
    d.n, d.b = sys_.n, sys_.b
    for k, v in enumerate((sys_.L1, sys_.L2, sys_.L3)):
        d.L[k] = v
    per = list(sys_.periodic) + [False] * (3 - sys_.crystal.D)
    for k in range(3):
        d.periodic[k] = int(per[k])
    d.acceptance = 1 if sys_.acceptance == "barker" else 0
    if sys_.h is not None:
        for k in range(sys_.n):
            d.h[k] = float(np.float32(sys_.h[k]))
    d.has_cubic = int(sys_.cubic_k1 is not None)
    d.k2 = float(np.float32(sys_.cubic_k2))
    col = sys_.colouring
    d.r = len(col.m)
    for r, mr in enumerate(col.m):
        d.m[r] = mr
        for k in range(sys_.crystal.D):
            d.K[r][k] = col.K[r][k] % mr
        for a in range(sys_.b):
            d.o[a][r] = col.o[a][r] % mr
    cl = classes(sys_)
    d.n_classes = len(cl)
    for i, (c, a) in enumerate(cl):
        d.classes[i][0], d.classes[i][1] = c, a
    bonds = sys_.crystal.bonds
    for a in range(sys_.b):
        groups, extras = field_groups(sys_, a)
        nb, g = 0, 0
        for J, members in groups.items():
            if J == 0.0 and not any(i in sys_.extra for i in members):
                continue
            for i in members:
                bd = bonds[i]
                dl = list(bd.delta) + [0] * (3 - sys_.crystal.D)
                e = d.bonds[a][nb]
                e.a2, e.dx, e.dy, e.dz = bd.alpha2, dl[0], dl[1], dl[2]
                e.extra = extras.index(i) if i in sys_.extra else -1
                nb += 1
            d.group_end[a][g] = nb
            d.J[a][g] = float(np.float32(J))
            d.apply[a][g] = int(J != 0.0)
            g += 1
        d.n_bonds[a], d.n_groups[a], d.n_extra[a] = nb, g, len(extras)
        for s, i in enumerate(extras):
            E = np.asarray(sys_.extra[i], np.float64)
            for k in range(sys_.n):
                for l in range(sys_.n):
                    d.E[a][s][3 * k + l] = float(np.float32(E[k, l]))
    return d


def ising_exp_table(sys_, beta: np.ndarray):
    """Every argument of exp an Ising chain of this system can reach, per replica, sorted, with NumPy's float32
    exp of each: (xs, es, offsets). The local field is enumerated with the port's float32 operation order
    (applied coupling groups, then extra bonds, then the field) over every neighbour sum a group can take
    (masks and open boundaries included) and every value an extra bond's neighbour can take; the argument is
    -beta dE (Metropolis) or beta dE (Barker) with dE = -((-s) - s) v."""
    f32 = np.float32
    vals = []
    for a in range(sys_.b):
        groups, extras = field_groups(sys_, a)
        axes = []
        coef = []
        for J, members in groups.items():
            if J == 0.0:
                continue
            z = len(members)
            axes.append(np.arange(-z, z + 1, dtype=np.float32))
            coef.append(("J", f32(J)))
        for i in extras:
            c = f32(np.asarray(sys_.extra[i], np.float64)[0, 0])
            if c != 0.0:
                axes.append(np.array([-1.0, 0.0, 1.0], np.float32))
                coef.append(("E", c))
        grids = np.meshgrid(*axes, indexing="ij") if axes else []
        v = np.zeros(grids[0].shape if grids else (1,), np.float32)
        for (kind, c), G in zip(coef, grids):
            v = (v + (c * G).astype(np.float32)).astype(np.float32)
        if sys_.h is not None and f32(sys_.h[0]) != 0.0:
            v = (v + f32(sys_.h[0])).astype(np.float32)
        vals.append(v.reshape(-1))
    v = np.unique(np.concatenate(vals))
    dEs = []
    for s in (f32(-1.0), f32(1.0)):
        acc_sum = ((-s - s) * v).astype(np.float32)
        dEs.append((-acc_sum).astype(np.float32))
    dE = np.unique(np.concatenate(dEs))
    xs, es, off = [], [], [0]
    barker = sys_.acceptance == "barker"
    for b in np.asarray(beta, np.float32):
        x = np.unique(((b if barker else -b) * dE).astype(np.float32))
        xs.append(x)
        es.append(np.exp(x).astype(np.float32))
        off.append(off[-1] + x.size)
    return np.concatenate(xs), np.concatenate(es), np.asarray(off, np.int64)


def sweep(sys_, S: np.ndarray, beta: np.ndarray, state: list[int], n: int = 1, reps=None, nthreads: int = 0):
    """n sweeps in place on float32 spins S (B, n, b, L3, L2, L1); state advances by n. Ising chains read exp from
    ising_exp_table (NumPy's values, as the reference's CPU path) and are bit-exact."""
    L = _load()
    S = np.ascontiguousarray(S, dtype=np.float32)
    B = S.shape[0]
    beta = np.ascontiguousarray(beta, dtype=np.float32)
    k1 = None if sys_.cubic_k1 is None else np.ascontiguousarray(sys_.cubic_k1, dtype=np.float32)
    mask = None if sys_.mask is None else np.ascontiguousarray(sys_.site_mask(), dtype=np.int8)
    r = None if reps is None else np.ascontiguousarray(reps, dtype=np.int64)
    d = describe(sys_)
    tab = ising_exp_table(sys_, beta) if sys_.n == 1 else None
    rc = L.oracle_sweep(ctypes.byref(d), S.ctypes.data, beta.ctypes.data, None if k1 is None else k1.ctypes.data,
                        None if mask is None else mask.ctypes.data, B, None if r is None else r.ctypes.data,
                        int(state[0]), int(state[1]), int(n), int(nthreads),
                        *((None, None, None) if tab is None else (t.ctypes.data for t in tab)))
    if rc != 0:
        raise RuntimeError("an Ising exp argument fell outside the enumerated table")
    state[1] += n
    return S


def bitwise_sweep(sys_, spins: np.ndarray, table: np.ndarray, base_seed: int, sweep0: int, n: int = 1,
                  independent: bool = False, words=None, nthreads: int = 0) -> np.ndarray:
    """n sweeps of the bitwise chain on unpacked spins (B, b, L3, L2, L1) of +-1 (0 masked); `words` gives the
    global word index of each block of 32 rows (default 0, 1, ...), `table` is indexed by local word: float32
    p_table (shared) or int64 p_fixed (independent). Returns the new spins (int8)."""
    from .bitwise import check
    L = _load()
    _, h, Z = check(sys_)
    S = np.ascontiguousarray(spins, dtype=np.int8).copy()
    B = S.shape[0]
    tab = np.ascontiguousarray(table, dtype=np.int64 if independent else np.float32)
    if tab.shape[-1] != Z + 1:
        raise ValueError("table does not match the system's coordination")
    mask = None if sys_.mask is None else np.ascontiguousarray(sys_.site_mask(), dtype=np.int8)
    w = None if words is None else np.ascontiguousarray(words, dtype=np.int64)
    d = describe(sys_)
    L.oracle_bitwise_sweep(ctypes.byref(d), S.ctypes.data, None if mask is None else mask.ctypes.data, B,
                           None if w is None else w.ctypes.data, tab.ctypes.data, Z + 1, int(h != 0.0),
                           int(independent), int(base_seed), int(sweep0), int(n), int(nthreads))
    return S


def time_heisenberg(sys_, T: np.ndarray, budget_s: float = 15.0, sweeps: int = 1, replicas: int | None = None,
                    warmup: int = 1, reps: int | None = None):
    """Attempts/ns of the C port on all host threads, in steady state: `replicas` replicas (default one per
    thread) of the full lattice, `sweeps` sweeps per repetition; `warmup` untimed repetitions (thread start-up,
    first touch of the spins), then `reps` timed repetitions, or as many as fit `budget_s` seconds (at least one).
    The CPU baseline and the reference arm of bench.py both report this rate."""
    nth = threads()
    R = replicas or nth
    g = np.random.default_rng(2)
    S = g.standard_normal((R, sys_.n) + sys_.shape).astype(np.float32)
    S /= np.linalg.norm(S, axis=1, keepdims=True)
    rows = np.arange(R, dtype=np.int64) * (len(T) // R if len(T) >= R else 1)
    beta = (np.float32(1.0) / np.asarray(T, np.float32)[rows % len(T)]).astype(np.float32)
    state = [1234, 0]
    for _ in range(warmup):
        sweep(sys_, S, beta, state, sweeps, reps=rows, nthreads=nth)
    t0 = time.perf_counter()
    done = n_rep = 0
    while True:
        sweep(sys_, S, beta, state, sweeps, reps=rows, nthreads=nth)
        done += R * sys_.n_active * sweeps
        n_rep += 1
        el = time.perf_counter() - t0
        if (reps is not None and n_rep >= reps) or (reps is None and el >= budget_s):
            break
    return {"value": done / (el * 1e9), "unit": "attempts/ns", "cores": nth, "kind": "port",
            "sample": f"C port (oracle/cpu_sweep.c, OpenMP, {nth} threads): {R} replicas x {sweeps} sweep(s) of the "
                      f"full {sys_.nsite}-site lattice per repetition, {warmup} untimed + {n_rep} timed "
                      f"repetitions ({el:.1f} s)"}


if __name__ == "__main__":
    print(build(force=True))
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
