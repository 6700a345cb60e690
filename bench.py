#!/usr/bin/env python
"""Throughput of the colour-class Metropolis sweep on B200: spin-update attempts per ns.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

One step = one sweep (every colour class of every replica) of the workload, inputs resident in HBM. The
default workload is the 3D Heisenberg bcc colour sweep: 64^3 cells x 2 sites (524,288 sites), J1 = 1, J2 = 0.3,
cubic K1 = 0.05, h = 0.1 along z, periodic, 64 replicas x 24 temperatures in [0.5, 2.5] (1,536 replicas,
9.66 GB of float32 state: larger than L2, so no flush is needed between steps); fp32 unit vectors uniform on
the sphere from seed 2 (drawn on the device), Philox key 1234 (+100000 per rank).

Multi-GPU (torchrun, one rank per GPU): every rank sweeps its own 1,536 replicas (replicas shard with no
exchange: weak scaling); the timed region is bracketed by barriers and the time is the max over ranks.

The JSON line carries the device-timed `value`, an end-to-end `e2e` figure through the public Sampler API
(per step: temperatures copied in from pinned host memory, the sweep, the FP64 observables and their copy back
to the host), the HBM roofline of the dominant kernel (algorithmic bytes: 24 B per attempt = 3 float32 read +
3 written), the sampled clocks, and the CPU baseline (the oracle port on the host cores).

--impl reference times the reference's CPU path on the host: the reference itself is Python that generates
Triton kernels and cannot travel to the GPU box, so its arithmetic is timed through the oracle port
(oracle/cpu_sweep.c, all host threads; the NumPy restatement when the C port is not built).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

RESIDENT_LIMIT = 200 << 10        # the plan's default: replicas up to 200 KiB sweep resident in shared memory
BYTES_PER_ATTEMPT = {"heisenberg-bcc": 24, "ising-sc-bitwise": 0.25, "ising-square": 2, "xy-ragged": 16,
                     "learned-ising-sc": 2}
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------------------------------------------ workloads
def heisenberg_bcc(L=64):
    from spin_colour_kernel_b200 import crystals as cr
    from spin_colour_kernel_b200 import system as sy
    c = cr.make("bcc", (1, 2))
    return sy.System("Heisenberg bcc J1-J2", 3, c, (L, L, L), (True,) * 3, {1: 1.0, 2: 0.3}, h=(0.0, 0.0, 0.1),
                     cubic_k1=np.full((2, L, L, L), 0.05, np.float32))


def make_workload(name, rank, device, L=64, replicas=1536, layout="quad"):
    from spin_colour_kernel_b200 import system as sy
    from spin_colour_kernel_b200.sampler import Sampler
    g = torch.Generator(device=device).manual_seed(2 + rank)
    if name == "heisenberg-bcc":
        s = heisenberg_bcc(L)
        B = replicas
        A = Sampler(s, B, device=device, seed=1234 + 100000 * rank, layout=layout)
        T = torch.linspace(0.5, 2.5, 24).repeat_interleave(-(-B // 24))[:B]
        S = torch.randn((B, 3) + s.shape, device=device, generator=g)
        S = (S / S.norm(dim=1, keepdim=True)).contiguous()
        if A.quad:
            S = A.pack(S)
        gb = B * 3 * s.nsite * 4 / 1e9
        cfg = {"workload": f"heisenberg-bcc-{L}^3x2-J1J2-K1-hz", "replicas": B, "sites": s.nsite,
               "temperatures": f"24 linear in [0.5, 2.5], {-(-B // 24)} replicas each", "spin_dtype": "float32",
               "layout": layout,
               "l2": f"no flush: {gb:.2f} GB state > 126 MB L2"}
    elif name == "ising-sc-bitwise":
        s = sy.ising("sc", 128)
        B = 512                                   # one counter-legal instance of the 1024-replica workload
        A = Sampler(s, B, device=device, seed=1 + 100000 * rank, bitwise=True)
        T = torch.linspace(4.0, 5.0, 16)[:8].repeat_interleave(64)
        S = A.pack(torch.randint(0, 2, (B, 1) + s.shape, device=device, generator=g, dtype=torch.int8) * 2 - 1)
        cfg = {"workload": "ising-sc-128^3-bitwise-shared", "replicas": B, "sites": s.nsite,
               "l2": "no flush: 128 MiB words ~ L2 size"}
    elif name == "ising-square":
        s = sy.ising("square", 32)
        B = 32
        A = Sampler(s, B, device=device, seed=1234 + 100000 * rank, packed=False)
        T = torch.tensor([1.5, 2.0, 2.269, 3.0]).repeat_interleave(8)
        S = A.init_spins(seed=0)
        cfg = {"workload": "ising-square-32^2-int8", "replicas": B, "sites": s.nsite, "l2": "resident (32 KB)"}
    else:
        raise SystemExit(f"unknown workload {name}")
    A.set_temperature(T)
    return s, A, S, T, cfg


# ------------------------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.out = None
        try:
            ident = str(torch.cuda.get_device_properties(device_index).uuid)
            ident = ident if ident.startswith("GPU-") else f"GPU-{ident}"
        except Exception:
            ident = str(device_index)
        self.ident = ident

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", self.ident, "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(kernel_tag):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, or None."""
    f = ROOT / "profiles" / f"{kernel_tag}.traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


# ---------------------------------------------------------------------------------------------- CPU side
def cpu_baseline(name, budget_s=15.0):
    """The oracle port on the host cores over a bounded sample of the workload: (attempts/ns, cores, kind,
    sample)."""
    from oracle import native
    if name != "heisenberg-bcc":
        return None
    s = heisenberg_bcc(64)
    T = torch.linspace(0.5, 2.5, 24).repeat_interleave(64).numpy()
    if native.available():
        return native.time_heisenberg(s, T, budget_s)
    from oracle import sweep as osw
    g = np.random.default_rng(2)
    x = g.standard_normal((1, 3) + s.shape).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    beta = np.asarray([np.float32(1.0) / np.float32(T[0])], np.float32)
    t0 = time.perf_counter()
    osw.sweep(s, x, beta, [1234, 0], 1, reps=[0])
    dt = time.perf_counter() - t0
    return {"value": s.nsite / (dt * 1e9), "unit": "attempts/ns", "cores": 1, "kind": "port",
            "sample": "NumPy oracle: 1 replica x 1 sweep of the full 64^3 x 2 bcc lattice"}


def reference_arm(args, rank, world):
    """The reference's CPU arithmetic for this path on the host cores: the oracle's C port (the reference itself is
    Python generating Triton kernels and cannot travel to the GPU box), W untimed and K timed repetitions of
    one sweep of one replica per host thread over the full lattice; the same steady-state rate as the
    `cpu_baseline` leg of the default arm."""
    if rank != 0:
        return
    s = heisenberg_bcc(64)
    T = torch.linspace(0.5, 2.5, 24).repeat_interleave(64).numpy()
    from oracle import native
    if native.available():
        base = native.time_heisenberg(s, T, warmup=max(1, args.warmup), reps=max(1, args.steps))
    else:
        base = cpu_baseline(args.workload)
    v = base["value"]
    cfg = {"workload": "heisenberg-bcc-64^3x2-J1J2-K1-hz", "replicas": 1536, "sites": s.nsite}
    line = {"impl": "reference", "metric": "spin-update attempts/ns", "value": v, "unit": "attempts/ns",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": "attempts/ns", "cores": base["cores"], "kind": base["kind"],
                             "sample": base["sample"]},
            "e2e": {"value": v, "unit": "attempts/ns", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_triton_arm(args, rank, world):
    """The reference's own GPU path on this B200: its generated Triton class kernels, driven through its public
    Sampler (Sampler(...).graph(S, k) replays timed with CUDA events, as its exp_perf.rate times them), from the
    unmodified package installed in baseline/_ref; none of this repository's kernels is loaded. Same workloads as
    this repository's arm: `heisenberg-bcc` (64^3 x 2, J1-J2, K1, h_z, 1,536 replicas at 24 temperatures; spins
    uniform on the sphere drawn on the device), `ising-square` (32^2, 32 int8 replicas) and `ising-sc-bitwise`
    (128^3, 512 replicas in shared-draw bitwise words). Prints the `unavailable` line with the reason when the
    package or its Triton compilation is missing here."""
    if rank != 0:
        return
    import tempfile
    ref = ROOT / "baseline" / "_ref"
    base = {"impl": "reference-triton", "metric": "spin-update attempts/ns", "unit": "attempts/ns"}
    if not (ref / "Spin_Colour_Kernel").is_dir():
        print(json.dumps({**base, "unavailable": "reference not installed in baseline/_ref"}), flush=True)
        return
    os.environ.setdefault("SCK_CACHE", tempfile.mkdtemp(prefix="sck_ref_cache_"))
    sys.path.insert(0, str(ref))
    try:
        from Spin_Colour_Kernel import crystals as rcr
        from Spin_Colour_Kernel import system as rsy
        from Spin_Colour_Kernel.sampler import Sampler as RefSampler
        device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(device)
        L, B = args.L, args.replicas
        g = torch.Generator(device=device).manual_seed(2)
        if args.workload == "ising-square":
            s = rsy.ising("square", 32)
            B = 32
            A = RefSampler(s, B, device, 1234, packed=False)
            A.set_temperature(torch.tensor([1.5, 2.0, 2.269, 3.0]).repeat_interleave(8))
            S = A.init_spins(seed=0)
            workload, dtype, sites = "ising-square-32^2-int8", "i8", int(s.n_active)
        elif args.workload == "ising-sc-bitwise":
            s = rsy.ising("sc", 128)
            B = 512
            A = RefSampler(s, B, device, 1, bitwise=True)
            A.set_temperature(torch.linspace(4.0, 5.0, 16)[:8].repeat_interleave(64))
            S = A.pack(torch.randint(0, 2, (B, 1) + s.shape, device=device, generator=g, dtype=torch.int8) * 2 - 1)
            workload, dtype, sites = "ising-sc-128^3-bitwise-shared", "u32", int(s.n_active)
        elif args.workload == "heisenberg-bcc":
            s = rsy.System("Heisenberg bcc J1-J2", 3, rcr.make("bcc", (1, 2)), (L, L, L), (True,) * 3,
                           {1: 1.0, 2: 0.3}, h=(0.0, 0.0, 0.1), cubic_k1=np.full((2, L, L, L), 0.05, np.float32))
            A = RefSampler(s, B, device, 1234)
            A.set_temperature(torch.linspace(0.5, 2.5, 24).repeat_interleave(-(-B // 24))[:B])
            S = torch.randn((B, 3) + s.shape, device=device, generator=g)
            S = (S / S.norm(dim=1, keepdim=True)).contiguous()
            workload, dtype, sites = f"heisenberg-bcc-{L}^3x2-J1J2-K1-hz", "f32", 2 * L ** 3
        else:
            print(json.dumps({**base, "unavailable": f"no reference-triton form of workload {args.workload}"}),
                  flush=True)
            return
        replay = A.graph(S, 1)
        for _ in range(max(1, args.warmup)):
            replay()
        torch.cuda.synchronize(device)
        clocks = ClockSampler(device.index)
        clocks.start()
        time.sleep(0.25)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            replay()
        e1.record()
        torch.cuda.synchronize(device)
        clk = clocks.stop()
        ms = e0.elapsed_time(e1)
    except Exception as exc:                     # no Triton for this GPU, a compile failure, ...
        print(json.dumps({**base, "unavailable": f"{type(exc).__name__}: {str(exc).splitlines()[0][:200]}"}),
              flush=True)
        return
    value = B * s.n_active * args.steps / (ms * 1e6)
    peak, kind = hbm_peak()
    bpa = BYTES_PER_ATTEMPT[args.workload]
    achieved = value * bpa
    loaded = sorted({m.__name__.split(".")[0] for m in list(sys.modules.values()) if m is not None and
                     getattr(m, "__name__", "").startswith(("spin_colour_kernel_b200", "Spin_Colour_Kernel"))})
    line = {**base, "value": value, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype, "data": "synthetic",
            "config": {"workload": workload, "replicas": B, "sites": sites,
                       "path": "reference Sampler.graph(S, 1) replays (generated Triton class kernels)",
                       "python_packages_loaded": loaded},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "note": f"algorithmic {bpa} B/attempt over the replay; peak {kind}"},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def ragged(args, rank, world, device):
    """96 XY systems of uneven size and mask in one batch, sweeps captured in a CUDA graph of 100 sweeps (or
    of K when K is not a multiple of 100); one step = one sweep of every system."""
    import torch.distributed as tdist
    from spin_colour_kernel_b200 import workloads as W
    from spin_colour_kernel_b200.sampler import Sampler
    rng = np.random.default_rng(3 + rank)
    samplers, spins = [], []
    attempts = 0
    for i, (crystal, L, disk, T) in enumerate(W.xy_ragged_specs()):
        s = W.xy_system(crystal, L, disk)
        A = Sampler(s, 32, device=device, seed=1234 + i + 100000 * rank)
        A.set_temperature(T)
        samplers.append(A)
        spins.append(torch.from_numpy(W.xy_angles(s, 32, rng)).to(device))
        attempts += 32 * s.n_active
    from spin_colour_kernel_b200.autotune import autotune_batch
    batch, tuned = autotune_batch(samplers, spins, use_cache=False)       # untimed: picks the resident limit
    G = 100 if args.steps % 100 == 0 else args.steps
    rep = batch.graph(G)
    for _ in range(max(1, args.warmup // G)):
        rep()
    torch.cuda.synchronize(device)
    if world > 1:
        tdist.barrier()
    clocks = ClockSampler(device.index)
    clocks.start()
    time.sleep(0.25)
    stream = torch.cuda.current_stream(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps // G):
        rep()
    e1.record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        x = torch.tensor([ms], device=device)
        tdist.all_reduce(x, op=tdist.ReduceOp.MAX)
        ms = float(x.item())
    info = batch.info()
    value = world * attempts * args.steps / (ms * 1e6)
    peak, kind = hbm_peak()
    achieved = attempts * 16 / ((ms / args.steps) * 1e-3) / 1e9
    line = {"metric": "spin-update attempts/ns", "value": value, "unit": "attempts/ns", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "xy-ragged-96 (48 square + 48 triangular, L log-uniform 16..512, half nanodisk)",
                       "systems": len(samplers), "replicas_per_system": 32, "attempts_per_sweep": attempts,
                       "graph_sweeps": G, "resident_systems": info["resident_systems"],
                       "autotune": {"resident_limit": tuned["resident_limit"], "tried": tuned["tried"]},
                       "l2": "no flush: state ~0.8 GB > L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "note": f"algorithmic 16 B/attempt over the whole step; peak {kind}"},
            "gpu_launches": 2 * (args.steps // G), "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------ learned block proposal
def learned(args, rank, world, device):
    """3D Ising sc L=64 periodic at T = 4.5115, 256 replicas: plain colour sweeps against block rounds of the
    learned proposal (8 colour steps of 4x4x4 blocks, MADE 160-256-256-256-64) plus one plain sweep. The network
    is trained on the 2^20 blocks of a plain-chain configuration of all replicas. Reports tau_int of |M| and E
    (Sokal window over the (time, replica) series) and effective independent samples per second of each arm."""
    from spin_colour_kernel_b200 import stats
    from spin_colour_kernel_b200 import system as sy
    from spin_colour_kernel_b200.learned import BlockProposal
    from spin_colour_kernel_b200.sampler import Sampler
    L, R, T = 64, 256, 4.5115
    K_plain, K_learned = args.learned_plain_sweeps, args.learned_rounds
    s = sy.ising("sc", L)
    A = Sampler(s, R, device=device, seed=5 + 1000 * rank, packed=False)
    A.set_temperature(torch.full((R,), T))
    S = A.init_spins(seed=1)
    A.sweep(S, args.learned_therm)
    beta = torch.full((R,), 1.0 / T, dtype=torch.float32, device=device)
    P = BlockProposal(L, R, groups=args.learned_groups, seed=7, device=device)
    ev = lambda: torch.cuda.Event(enable_timing=True)          # noqa: E731
    t0, t1 = ev(), ev()
    t0.record()
    data = P.gather(S)
    losses = P.train(data, steps=args.learned_train_steps, batch=8192, lr=1e-3)
    t1.record()
    torch.cuda.synchronize(device)
    train_ms = t0.elapsed_time(t1)
    del data

    def series(step, K):
        X = S.clone()
        E_all = torch.empty((K, R), dtype=torch.float64, device=device)
        M_all = torch.empty((K, R), dtype=torch.float64, device=device)
        E = torch.empty(R, dtype=torch.float64, device=device)
        M = torch.empty((R, 1, 1), dtype=torch.float64, device=device)
        for k in range(K):
            step(X, k)
            A.observables(X, E, M)
            E_all[k].copy_(E)
            M_all[k].copy_(M.reshape(R).abs())
        return E_all.cpu().numpy() / L ** 3, M_all.cpu().numpy() / L ** 3, X

    def timed(step, K):
        X = S.clone()
        for k in range(3):
            step(X, k)
        torch.cuda.synchronize(device)
        a, b = ev(), ev()
        a.record()
        for k in range(K):
            step(X, k)
        b.record()
        torch.cuda.synchronize(device)
        return a.elapsed_time(b) / K

    acc = torch.zeros(R, dtype=torch.int32, device=device)

    def plain_step(X, k):
        A.sweep(X, 1)

    def learned_step(X, k):
        P.round(X, beta, seed=11, rnd=k, accepted=acc)
        A.sweep(X, 1)

    clocks = ClockSampler(device.index)
    clocks.start()
    ms_plain = timed(plain_step, 200)
    ms_learned = timed(learned_step, 50)
    clk = clocks.stop()
    acc.zero_()
    Ep, Mp, _ = series(plain_step, K_plain)
    El, Ml, _ = series(learned_step, K_learned)
    acceptance = float(acc.sum().item()) / (K_learned * R * (L // 4) ** 3)
    out = {}
    for name, (E_, M_, ms) in {"plain": (Ep, Mp, ms_plain), "learned": (El, Ml, ms_learned)}.items():
        tm, te = stats.integrated_tau(M_), stats.integrated_tau(E_)
        rate = R / (ms * 1e-3)                     # configurations (replica steps) per second
        out[name] = {"ms_per_step": ms, "tau_int_absM": tm, "tau_int_E": te, "steps": int(E_.shape[0]),
                     "eff_samples_per_s_absM": stats.effective_rate(rate, tm),
                     "eff_samples_per_s_E": stats.effective_rate(rate, te),
                     "absM": [float(M_.mean()), float(M_.std() * np.sqrt(2 * tm / M_.size))],
                     "E": [float(E_.mean()), float(E_.std() * np.sqrt(2 * te / E_.size))]}
    agree = {k: abs(out["plain"][k][0] - out["learned"][k][0]) /
             max(np.hypot(out["plain"][k][1], out["learned"][k][1]), 1e-300) for k in ("absM", "E")}
    gain = out["learned"]["eff_samples_per_s_absM"] / out["plain"]["eff_samples_per_s_absM"]
    line = {"metric": "effective independent samples/s of |M| (learned block proposal)",
            "value": out["learned"]["eff_samples_per_s_absM"], "unit": "samples/s", "n_gpus": world,
            "higher_is_better": True, "vs_plain": gain, "dtype": "bf16/f32", "data": "synthetic",
            "config": {"workload": "learned-ising-sc-64 (T=4.5115, 256 replicas, 4x4x4 blocks, 8 colours)",
                       "groups": args.learned_groups, "therm_sweeps": args.learned_therm,
                       "train_steps": args.learned_train_steps, "train_batch": 8192, "train_blocks": R * 4096,
                       "train_ms": train_ms, "loss_first": float(losses[:10].mean()),
                       "loss_last": float(losses[-10:].mean())},
            "acceptance": acceptance, "plain": out["plain"], "learned": out["learned"],
            "agreement_sigma": agree, "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="heisenberg-bcc", choices=sorted(BYTES_PER_ATTEMPT))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-triton"],
                    help="ours; reference = the reference's CPU arithmetic on the host cores; reference-triton = "
                         "the reference's own Triton kernels on this GPU (installed in baseline/_ref)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--L", type=int, default=64, help="heisenberg-bcc cells per axis (profiling runs use less)")
    ap.add_argument("--replicas", type=int, default=1536, help="heisenberg-bcc replicas")
    ap.add_argument("--group", type=int, default=None,
                    help="interleaved layout: replicas per group of the class-skewed L2 pipeline (0 = class by class)")
    ap.add_argument("--skew", type=int, default=2, help="interleaved layout: class skew of the pipeline")
    ap.add_argument("--chunks", type=int, default=None, help="interleaved layout: site blocks per pipeline ticket")
    ap.add_argument("--layout", default="quad", choices=["quad", "reference"],
                    help="heisenberg-bcc resident storage: interleaved quads (default) or the reference layout")
    ap.add_argument("--path", default="auto",
                    choices=["auto", "autotune", "tile", "segment", "row", "lattice", "generic"],
                    help="sweep path: plan default, autotuned, tile kernels, segment kernels ('row' is an alias), "
                         "lattice kernels only, or generic kernels")
    ap.add_argument("--learned-groups", type=int, default=16, choices=[16, 64])
    ap.add_argument("--learned-therm", type=int, default=2000)
    ap.add_argument("--learned-train-steps", type=int, default=1000)
    ap.add_argument("--learned-plain-sweeps", type=int, default=6000)
    ap.add_argument("--learned-rounds", type=int, default=1500)
    ap.add_argument("--l2-mb", type=float, default=None,
                    help="L2 budget of the group pipeline (MiB); with an explicit --path, 0 (class by class) "
                         "unless given")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.impl == "reference-triton":
        reference_triton_arm(args, rank, world)
        return
    import datetime
    if dist:
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    from spin_colour_kernel_b200 import build as bld
    bld.build()
    if args.workload in ("xy-ragged", "learned-ising-sc"):
        (ragged if args.workload == "xy-ragged" else learned)(args, rank, world, device)
        if dist:
            tdist.barrier()
            tdist.destroy_process_group()
        return
    s, A, S, T, cfg = make_workload(args.workload, rank, device, args.L, args.replicas, args.layout)
    budget = int((args.l2_mb or 0) * (1 << 20))
    if A.quad:
        if args.group:
            A.pipeline(args.group, args.skew, args.chunks)
        cfg["pipeline"] = {"group": A.path()["group"], "skew": args.skew if args.group else None,
                           "chunks": (args.chunks or 4) if args.group else None}
    elif args.path in ("tile", "segment", "row", "lattice", "generic"):
        A.tune({"tile": 3, "segment": 2, "row": 2, "lattice": 1, "generic": 0}[args.path], budget, RESIDENT_LIMIT)
    elif args.path == "autotune":
        from spin_colour_kernel_b200.autotune import autotune
        cfg["autotune"] = autotune(A, S, use_cache=False)
    elif args.l2_mb is not None:
        A.tune(1, budget, RESIDENT_LIMIT)
    attempts_per_step = A.B * s.n_active
    stream = torch.cuda.current_stream(device)
    classes = list(A.classes)
    path = A.path()
    C = len(classes)
    groups = -(-A.Bp // path["group"]) if path["group"] else 0
    # the K timed steps are one call sweep(S, K): the library sees the whole sequence (a resident launch runs all
    # K sweeps on-chip, the L2 pipeline overlaps consecutive sweeps), as a user running K sweeps would call it
    K = args.steps
    if path["resident"] or (A.quad and groups):
        launches = 1                       # one resident launch, or one pipeline launch, per call of K sweeps
    elif groups:
        launches = K * groups + C - 1
    else:
        launches = K * C * (-(-A.Bp // (65535 * (2 if s.n > 1 else 1))))

    for _ in range(args.warmup):
        A.sweep(S, 1)
    torch.cuda.synchronize(device)
    if dist:
        tdist.barrier()
    clocks = ClockSampler(device.index)
    clocks.start()
    time.sleep(0.25)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    A.sweep(S, K)
    ev[1].record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    ms = ev[0].elapsed_time(ev[1])
    step_ms = [ms / K]
    if dist:
        x = torch.tensor([ms], device=device)
        tdist.all_reduce(x, op=tdist.ReduceOp.MAX)
        ms = float(x.item())
        tdist.barrier()

    # end to end through the public API: temperatures in from pinned host memory, one measure step (a sweep and
    # the FP64 observables of the state it leaves), observables out to pinned host memory, every step
    beta_h = (1.0 / T).to(torch.float32).pin_memory()
    E = torch.empty(A.B, dtype=torch.float64, device=device)
    M = torch.empty((A.B, s.b, s.n), dtype=torch.float64, device=device)
    E_h = torch.empty(A.B, dtype=torch.float64).pin_memory()
    M_h = torch.empty((A.B, s.b, s.n), dtype=torch.float64).pin_memory()
    e2e_steps = max(3, args.steps // 2)
    A.sweep_measure(S, 1, E, M)          # untimed: sizes the measure step's workspace
    torch.cuda.synchronize(device)
    if dist:
        tdist.barrier()
    u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    u0.record(stream)
    for _ in range(e2e_steps):
        A.beta[: A.B].copy_(beta_h, non_blocking=True)
        A.sweep_measure(S, 1, E, M)
        E_h.copy_(E, non_blocking=True)
        M_h.copy_(M, non_blocking=True)
    u1.record(stream)
    torch.cuda.synchronize(device)
    e2e_ms = u0.elapsed_time(u1)
    if dist:
        x = torch.tensor([e2e_ms], device=device)
        tdist.all_reduce(x, op=tdist.ReduceOp.MAX)
        e2e_ms = float(x.item())

    value = world * attempts_per_step * args.steps / (ms * 1e6)
    e2e = world * attempts_per_step * e2e_steps / (e2e_ms * 1e6)
    bpa = BYTES_PER_ATTEMPT[args.workload]
    # the timed launches run back to back on one stream: their mean duration is the timed region over the launches
    # (inter-launch gaps and the counter updates included, so this is a lower bound on the kernel's rate)
    launches_per_sweep = launches / K
    bytes_per_launch = attempts_per_step * K * bpa / launches
    mean_launch_ms = ms / launches
    achieved = bytes_per_launch / (mean_launch_ms * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    traffic = traffic_per_launch(f"{args.workload}" + ("-quad" if A.quad else ""))
    line = {
        "metric": "spin-update attempts/ns", "value": value, "unit": "attempts/ns", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if s.n > 1 else "u32", "data": "synthetic",
        "config": cfg,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "note": f"algorithmic {bpa} B/attempt; peak {peak_kind}; kernel = "
                             f"{'bitwise' if A.bitwise else ['generic', 'lattice', 'segment', 'tile', 'interleaved'][path['specialised'] // 100]} class update, "
                             f"{launches_per_sweep} launches per sweep (L2 group {path['group']}), "
                             f"step times from CUDA events"},
        "e2e": {"value": e2e, "unit": "attempts/ns", "h2d_bytes_per_step": int(beta_h.numel() * 4),
                "d2h_bytes_per_step": int((E_h.numel() + M_h.numel()) * 8)},
        "gpu_launches": int(launches + (1 if path["resident"] or groups else K)),
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
