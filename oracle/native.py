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
                                   ctypes.c_void_p, _i32, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, _i32, _i32]
        L.oracle_sweep.restype = _i32
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


def sweep(sys_, S: np.ndarray, beta: np.ndarray, state: list[int], n: int = 1, reps=None, nthreads: int = 0):
    """n sweeps in place on float32 spins S (B, n, b, L3, L2, L1); state advances by n."""
    L = _load()
    S = np.ascontiguousarray(S, dtype=np.float32)
    B = S.shape[0]
    beta = np.ascontiguousarray(beta, dtype=np.float32)
    k1 = None if sys_.cubic_k1 is None else np.ascontiguousarray(sys_.cubic_k1, dtype=np.float32)
    mask = None if sys_.mask is None else np.ascontiguousarray(sys_.site_mask(), dtype=np.int8)
    r = None if reps is None else np.ascontiguousarray(reps, dtype=np.int64)
    d = describe(sys_)
    L.oracle_sweep(ctypes.byref(d), S.ctypes.data, beta.ctypes.data, None if k1 is None else k1.ctypes.data,
                   None if mask is None else mask.ctypes.data, B, None if r is None else r.ctypes.data,
                   int(state[0]), int(state[1]), int(n), int(nthreads))
    state[1] += n
    return S


def time_heisenberg(sys_, T: np.ndarray, budget_s: float = 15.0, sweeps: int = 1, replicas: int | None = None):
    """Attempts/ns of the C port on all host threads: `replicas` replicas (default one per thread) of the full
    lattice, `sweeps` sweeps, repeated until `budget_s` seconds have passed (at least once)."""
    nth = threads()
    R = replicas or nth
    g = np.random.default_rng(2)
    S = g.standard_normal((R, sys_.n) + sys_.shape).astype(np.float32)
    S /= np.linalg.norm(S, axis=1, keepdims=True)
    reps = np.arange(R, dtype=np.int64) * (len(T) // R if len(T) >= R else 1)
    beta = (np.float32(1.0) / np.asarray(T, np.float32)[reps % len(T)]).astype(np.float32)
    state = [1234, 0]
    t0 = time.perf_counter()
    done = 0
    while True:
        sweep(sys_, S, beta, state, sweeps, reps=reps, nthreads=nth)
        done += R * sys_.n_active * sweeps
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return {"value": done / (el * 1e9), "unit": "attempts/ns", "cores": nth, "kind": "port",
            "sample": f"C port (oracle/cpu_sweep.c, OpenMP): {R} replicas x {sweeps} sweep(s) of the full "
                      f"{sys_.nsite}-site lattice per repetition, {el:.1f} s"}


if __name__ == "__main__":
    print(build(force=True))
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
