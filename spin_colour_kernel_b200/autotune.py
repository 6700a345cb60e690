"""Autotuner of the sweep's execution path.

The chain a Sampler produces does not depend on how its sweeps are executed, only the speed does. The knobs of
the plan (`sck_plan_tune`) are: the specialised lattice kernels on or off, and the L2 budget of the group
pipeline (0 = class by class over all replicas). `autotune(sampler, S)` times every candidate on a scratch copy
of the spins with CUDA events, keeps the fastest, restores the sweep counter, and caches the choice per
(system, batch, mode, device) in a JSON file (`$SCK_TUNE_CACHE`, default ~/.cache/spin_colour_kernel_b200/).
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


def candidates(sampler):
    """(specialised, l2_budget, resident_limit) triples worth timing for this sampler."""
    out = [(0, 0, 0), (0, 0, RESIDENT_LIMIT)]
    kind = sampler.tune(2, 0, 0)["specialised"] // 100
    for level in range(1, kind + 1):
        out += [(level, mb << 20, 0) for mb in CANDIDATE_BUDGETS_MB]
    return out


def autotune(sampler, S: torch.Tensor, sweeps: int = 3, use_cache: bool = True) -> dict:
    """Pick and apply the fastest path for this sampler; returns {"specialised", "l2_budget", "ms", ...}."""
    key = system_key(sampler)
    cache = _load() if use_cache else {}
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
        sampler.sweep(work, 1)                         # warm-up
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream(sampler.device)
        a.record(stream)
        sampler.sweep(work, sweeps)
        b.record(stream)
        torch.cuda.synchronize(sampler.device)
        results.append((a.elapsed_time(b) / sweeps, spec, budget, resident, p))
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


__all__ = ["autotune", "candidates", "system_key", "ms_table"]
