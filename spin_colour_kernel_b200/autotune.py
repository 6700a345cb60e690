"""Autotuner of the sweep's execution path.

The chain a Sampler produces does not depend on how its sweeps are executed, only the speed does. For the
reference layout the knobs of the plan (`sck_plan_tune`) are: the kernel level (generic, lattice, segment, tile),
the L2 budget of the group pipeline (0 = class by class over all replicas) and the resident limit. For the
interleaved ('quad') layout they are the class schedule of `sck_plan_pipeline`: class-by-class launches, or the
L2 pipeline with groups of 4, 8, 16 or 32 replicas, every class skew that divides the class count (the order
in which the classes of different groups run; a group's own classes always run in sweep order, so the chain is
unchanged) and 1 or 4 site blocks per pipeline ticket (`sck_plan_pipeline_chunks`). For a ragged batch
(`autotune_batch`) the knob is the resident limit: which systems run every sweep of a call on-chip and which
stream class by class through the persistent kernel. `autotune(sampler, S)` times every candidate on a scratch copy of the spins with CUDA events, keeps
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
QUAD_CHUNKS = (1, 4)


def quad_candidates(sampler):
    """(group replicas, skew, site blocks per ticket) of the interleaved layout: (0, 1, 4) = class by class."""
    C = len(sampler.classes)
    Q = sampler.Q
    out = [(0, 1, 4)]
    for g in QUAD_GROUPS:
        ngroups = -(-Q // min(g // 4, Q))
        for d in range(1, C + 1):
            if C % d == 0 and C <= 8 and d * ngroups >= C:
                out += [(g, d, c) for c in QUAD_CHUNKS]
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
    if key in cache and "chunks" in cache[key]:
        c = cache[key]
        sampler.pipeline(c["group"], c["skew"], c["chunks"])
        return dict(c, cached=True)
    saved = sampler.state.clone()
    work = S.clone()
    results = []
    for g, d, ch in quad_candidates(sampler):
        sampler.pipeline(g, d, ch)
        results.append((_time(sampler, work, sweeps), g, d, ch))
    sampler.check_waits()
    sampler.state.copy_(saved)
    del work
    ms, g, d, ch = min(results, key=lambda r: r[0])
    sampler.pipeline(g, d, ch)
    choice = {"layout": "quad", "group": g, "skew": d, "chunks": ch, "ms_per_sweep": ms,
              "tried": [{"group": r[1], "skew": r[2], "chunks": r[3], "ms": r[0]} for r in results]}
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


BATCH_RESIDENT_LIMITS = (0, 16 << 10, 48 << 10, 100 << 10, 200 << 10)


def batch_key(samplers) -> str:
    h = hashlib.sha256()
    for s in samplers:
        h.update(system_key(s).encode())
    return "batch:" + h.hexdigest()[:24]


def autotune_batch(samplers, spins, sweeps: int = 5, use_cache: bool = True):
    """A SamplerBatch of these samplers with the fastest resident limit, and the choice: each candidate batch is
    timed on scratch copies of the spins (CUDA events over `sweeps` sweeps after one warm-up sweep); the sweep
    counters are restored and the returned batch is bound to `spins`. Cached per set of systems."""
    from .sampler import SamplerBatch
    key = batch_key(samplers)
    cache = _load() if use_cache else {}
    if key in cache:
        c = cache[key]
        return SamplerBatch(samplers, spins, resident_limit=c["resident_limit"]), dict(c, cached=True)
    saved = [s.state.clone() for s in samplers]
    work = [S.clone() for S in spins]
    dev = samplers[0].device
    results, seen = [], set()
    for limit in BATCH_RESIDENT_LIMITS:
        b = SamplerBatch(samplers, work, resident_limit=limit)
        info = b.info()
        if info["resident_systems"] in seen:
            continue
        seen.add(info["resident_systems"])
        b.sweep(1)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream(dev)
        a.record(stream)
        b.sweep(sweeps)
        e.record(stream)
        torch.cuda.synchronize(dev)
        b.check_waits()
        results.append((a.elapsed_time(e) / sweeps, limit, info["resident_systems"]))
        del b
    for s, st in zip(samplers, saved):
        s.state.copy_(st)
    del work
    ms, limit, res = min(results, key=lambda r: r[0])
    choice = {"resident_limit": limit, "resident_systems": res, "ms_per_sweep": ms,
              "tried": [{"resident_limit": r[1], "resident_systems": r[2], "ms": r[0]} for r in results]}
    if use_cache:
        cache[key] = choice
        _store(cache)
    return SamplerBatch(samplers, spins, resident_limit=limit), dict(choice, cached=False)


def ms_table(results) -> str:
    rows = sorted(results, key=lambda r: r["ms"])
    return "\n".join(f"spec={r['specialised']} group={r['group']}: {r['ms']:.3f} ms" for r in rows)


__all__ = ["autotune", "autotune_batch", "candidates", "quad_candidates", "system_key", "batch_key", "ms_table"]
