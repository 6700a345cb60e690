"""Autotuner of the sweep's execution path.

The chain a Sampler produces does not depend on how its sweeps are executed, only the speed does. For the
reference layout the knobs of the plan (`sck_plan_tune`) are: the kernel level (generic, lattice, segment, tile),
the L2 budget of the group pipeline (0 = class by class over all replicas) and the resident limit. For the
interleaved ('quad') layout they are the class schedule of `sck_plan_pipeline`: class-by-class launches, or the
L2 pipeline with groups of 4, 8, 16 or 32 replicas and every class skew that divides the class count (the order
in which the classes of different groups run; a group's own classes always run in sweep order, so the chain is
unchanged). `autotune(sampler, S)` times every candidate on a scratch copy of the spins with CUDA events, keeps
the fastest, restores the sweep counter, and caches the choice per (system, batch, mode, device) in a JSON file
(`$SCK_TUNE_CACHE`, default ~/.cache/spin_colour_kernel_b200/).
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import torch

CANDIDATE_BUDGETS_MB = (0, 32, 48, 72, 96)


def _cache_file() -> Path:
    root = os.environ.get("SCK_TUNE_CACHE")
    return Path(root) if root else Path.home() / ".cache" / "spin_colour_kernel_b200" / "tune.json"


def system_key(sampler) -> str:
    """Hash of everything that shapes a sweep's work: the lowered descriptor, batch, mode and device name."""
    import ctypes
    h = hashlib.sha256(bytes(ctypes.string_at(ctypes.addressof(sampler.desc), ctypes.sizeof(sampler.desc))))
    h.update(f"{sampler.B}:{sampler.mode}:{torch.cuda.get_device_name(sampler.device)}".encode())
    return h.hexdigest()[:24]


def _load() -> dict:
    f = _cache_file()
    try:
        return json.loads(f.read_text())
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    f = _cache_file()
    try:
        f.parent.mkdir(parents=True, exist_ok=True)
        f.write_text(json.dumps(d, indent=1))
    except OSError:
        pass


RESIDENT_LIMIT = 200 << 10


QUAD_GROUPS = (4, 8, 16, 32)


def quad_candidates(sampler):
    """(group replicas, skew) pairs of the interleaved layout: (0, 1) = class by class."""
    C = len(sampler.classes)
    Q = sampler.Q
    out = [(0, 1)]
    for g in QUAD_GROUPS:
        ngroups = -(-Q // min(g // 4, Q))
        for d in range(1, C + 1):
            if C % d == 0 and C <= 8 and d * ngroups >= C:
                out.append((g, d))
    return out


def _time(sampler, work, sweeps):
    sampler.sweep(work, 1)                         # warm-up
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(sampler.device)
    a.record(stream)
    sampler.sweep(work, sweeps)
    b.record(stream)
    torch.cuda.synchronize(sampler.device)
    return a.elapsed_time(b) / sweeps


def _autotune_quad(sampler, S, sweeps, use_cache, key, cache):
    if key in cache:
        c = cache[key]
        sampler.pipeline(c["group"], c["skew"])
        return dict(c, cached=True)
    saved = sampler.state.clone()
    work = S.clone()
    results = []
    for g, d in quad_candidates(sampler):
        sampler.pipeline(g, d)
        results.append((_time(sampler, work, sweeps), g, d))
    sampler.check_waits()
    sampler.state.copy_(saved)
    del work
    ms, g, d = min(results, key=lambda r: r[0])
    sampler.pipeline(g, d)
    choice = {"layout": "quad", "group": g, "skew": d, "ms_per_sweep": ms,
              "tried": [{"group": r[1], "skew": r[2], "ms": r[0]} for r in results]}
    if use_cache:
        cache[key] = choice
        _store(cache)
    return dict(choice, cached=False)


def candidates(sampler):
    """(specialised, l2_budget, resident_limit) triples worth timing for this sampler (reference layout)."""
    out = [(0, 0, 0), (0, 0, RESIDENT_LIMIT)]
    kind = sampler.tune(2, 0, 0)["specialised"] // 100
    for level in range(1, kind + 1):
        out += [(level, mb << 20, 0) for mb in CANDIDATE_BUDGETS_MB]
    return out


def autotune(sampler, S: torch.Tensor, sweeps: int = 3, use_cache: bool = True) -> dict:
    """Pick and apply the fastest path for this sampler; returns {"specialised", "l2_budget", "ms", ...}."""
    key = system_key(sampler)
    cache = _load() if use_cache else {}
    if getattr(sampler, "quad", False):
        return _autotune_quad(sampler, S, sweeps, use_cache, key, cache)
    if key in cache:
        c = cache[key]
        sampler.tune(c["level"], c["l2_budget"], c["resident_limit"])
        return dict(c, cached=True)
    saved = sampler.state.clone()
    work = S.clone()
    results = []
    seen = set()
    for spec, budget, resident in candidates(sampler):
        p = sampler.tune(spec, budget, resident)
        sig = (p["specialised"], p["group"], p["resident"])
        if sig in seen:
            continue
        seen.add(sig)
        results.append((_time(sampler, work, sweeps), spec, budget, resident, p))
    sampler.state.copy_(saved)
    del work
    ms, spec, budget, resident, p = min(results, key=lambda r: r[0])
    sampler.tune(spec, budget, resident)
    choice = {"level": spec, "specialised": p["specialised"], "l2_budget": budget, "resident_limit": resident, "group": p["group"],
              "resident": p["resident"], "ms_per_sweep": ms,
              "tried": [{"specialised": r[4]["specialised"], "group": r[4]["group"], "resident": r[4]["resident"],
                         "ms": r[0]} for r in results]}
    if use_cache:
        cache[key] = choice
        _store(cache)
    return dict(choice, cached=False)


def ms_table(results) -> str:
    rows = sorted(results, key=lambda r: r["ms"])
    return "\n".join(f"spec={r['specialised']} group={r['group']}: {r['ms']:.3f} ms" for r in rows)


__all__ = ["autotune", "candidates", "quad_candidates", "system_key", "ms_table"]
