"""One state of a temperature ladder on the sm_100a library: the reference's `simulate.simulate_state`
(`src/Spin_Colour_Kernel/simulate.py:322-402`) with the same arguments, the same outputs and the same chain.

For each temperature (descending ladder, one chain per replica carried from one temperature to the next) the
runner thermalises, takes the FP64 energy of the state as a reference E_ref, then makes m = n_meas // every
observations, each after `every` sweeps. An observation adds, per replica, E - E_ref, (E - E_ref)^2, |m|,
|m|^2 and the mean magnetization vector m to FP64 accumulators; the results are
    E = E_ref + <E - E_ref>,  E2 = <(E - E_ref)^2> + 2 E_ref <E - E_ref> + E_ref^2,
    Mabs = <|m|>,  M2 = <|m|^2>,  M = <m> (float32, three components),
and every `config_every`-th temperature saves each replica's active-site spins.

Where the reference runs the observation as a chain of torch operations on an FP64 copy of the state
(`simulate.py:267-319`), here one library call does it: the observables pass (`sck_observables`) and a fold of
its result into the accumulators on the device (`sck_observables_accumulate`). The measure step — `every`
sweeps and that call — is captured once in a CUDA graph and replayed (packed Ising excepted, as in the
reference), and thermalisation replays a graph of 10 x `every` sweeps.
"""

from __future__ import annotations

import time

import numpy as np
import torch

from .sampler import Sampler
from .system import System


def temperature_ladder(T_max: float, T_min: float, T_step: float) -> np.ndarray:
    """Descending temperatures T_max, T_max - T_step, ..., down to T_min (`simulate.py:243-249`)."""
    hi, lo, step = float(T_max), float(T_min), float(T_step)
    if step <= 0 or lo <= 0 or hi < lo:
        raise ValueError("need T_max >= T_min > 0 and T_step > 0")
    count = int(np.floor((hi - lo) / step + 1e-9)) + 1
    return np.round(hi - step * np.arange(count), 10)


def site_spins(A: Sampler, S: torch.Tensor, mask: np.ndarray) -> np.ndarray:
    """(B, n_active, 3) float32 spins of the active sites in (b, z, y, x) order; missing components are 0."""
    x = A.unpack(S).float()                                   # (B, n, b, L3, L2, L1)
    B, n = x.shape[0], x.shape[1]
    flat = x.reshape(B, n, -1)[:, :, torch.from_numpy(mask.reshape(-1)).to(x.device)]
    out = np.zeros((B, flat.shape[2], 3), np.float32)
    out[:, :, :n] = flat.permute(0, 2, 1).cpu().numpy()
    return out


class _Measure:
    """Device buffers of one state's measurements and the calls that fill them."""

    def __init__(self, A: Sampler, S: torch.Tensor):
        s, dev = A.sys, A.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.A, self.S = A, S
        self.E_ref = torch.zeros(A.B, **f64)
        self.E = torch.zeros(A.B, **f64)
        self.M = torch.zeros((A.B, s.b, s.n), **f64)
        self.acc = torch.zeros((4, A.B), **f64)
        self.accv = torch.zeros((A.B, s.n), **f64)

    def reference(self):
        self.A.observables(self.S, self.E_ref, self.M)

    def clear(self):
        self.acc.zero_()
        self.accv.zero_()

    def step(self, every: int):
        self.A.sweep(self.S, every)
        self.A.observe(self.S, self.E_ref, self.acc, self.accv, self.E, self.M)


def simulate_state(s: System, replicas: int, temps, n_therm: int, n_meas: int, every: int, config_every: int,
                   seed: int, device="cuda", kB: float = 1.0, log=print, graphs: bool | None = None) -> dict:
    """Run the ladder `temps` for one system; energies are totals, M is the mean magnetization per site.

    Returns M (B, nT, 3) float32, E, E2, Mabs, M2 (B, nT) float64, configs (B, n_saved, n_active, 3) float32 and
    config_temperatures, as the reference does. `graphs=False` replays nothing (every launch from the host)."""
    A = Sampler(s, int(replicas), device, seed)
    S = A.init_spins(seed=seed)
    mask = s.site_mask()
    every = max(1, int(every))
    n_obs = max(1, int(n_meas) // every)
    block = 10 * every
    ce = max(1, int(config_every))
    temps = np.asarray(temps, float)
    nT, B = len(temps), int(replicas)
    saved = [t for t in range(nT) if t % ce == 0]
    out = dict(M=np.zeros((B, nT, 3), np.float32), E=np.zeros((B, nT)), E2=np.zeros((B, nT)),
               Mabs=np.zeros((B, nT)), M2=np.zeros((B, nT)),
               configs=np.zeros((B, len(saved), int(mask.sum()), 3), np.float32),
               config_temperatures=temps[saved])
    meas = _Measure(A, S)
    use_graphs = (A.device.type == "cuda" and not A.packed) if graphs is None else bool(graphs)
    A.set_temperature(kB * float(temps[0]))
    if use_graphs:
        therm = A.graph(S, block)
        dev = A.device
        with torch.cuda.device(dev):
            side = torch.cuda.Stream(device=dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                meas.step(every)                          # warm-up (workspace, lazy state) outside the capture
            torch.cuda.current_stream(dev).wait_stream(side)
            torch.cuda.synchronize(dev)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                meas.step(every)

        def observe_step():
            with torch.cuda.device(dev):
                g.replay()
    else:
        def therm():
            A.sweep(S, block)

        def observe_step():
            meas.step(every)

    t0 = time.perf_counter()
    for t, T in enumerate(temps):
        A.set_temperature(kB * float(T))
        for _ in range(int(n_therm) // block):
            therm()
        if int(n_therm) % block:
            A.sweep(S, int(n_therm) % block)
        meas.reference()
        meas.clear()
        for _ in range(n_obs):
            observe_step()
        d, d2, ma, m2 = (meas.acc / n_obs).cpu().numpy()
        er = meas.E_ref.cpu().numpy()
        out["E"][:, t] = er + d
        out["E2"][:, t] = d2 + 2 * er * d + er * er
        out["Mabs"][:, t] = ma
        out["M2"][:, t] = m2
        out["M"][:, t, :s.n] = (meas.accv / n_obs).float().cpu().numpy()
        if t in saved:
            out["configs"][:, saved.index(t)] = site_spins(A, S, mask)
        if t % max(1, nT // 10) == 0 or t == nT - 1:
            log(f"    T = {T:9.4f}   <E>/site = {out['E'][:, t].mean() / s.n_active:+.4f}"
                f"   <|M|> = {out['Mabs'][:, t].mean():.4f}   {time.perf_counter() - t0:8.1f} s")
    return out
