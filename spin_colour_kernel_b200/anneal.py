"""Cooling ladder of the magnetic nanodisk on the sm_100a library: the reference's `anneal` module
(`src/Spin_Colour_Kernel/anneal.py`) with the same functions, arguments and outputs.

A state is one nanodisk Hamiltonian (seven parameters: Jex2, Jex3, Jex4, Kan1, KanS, Hex, KDM; Jex = 1 sets the
energy unit, temperatures in kelvin) and one batch of replicas that all follow the ladder T_start -> T_end. At
each temperature a replica thermalises, a reference (E_ref, |M|_ref) is taken, and every `every` sweeps an
observation adds dE = E - E_ref, dE^2, dM = |M| - |M|_ref, dM^2, M_z and the middle layer's Berg-Luscher
charge Q to FP64 accumulators; `reduce_obs` turns them into E, M, C_v, chi, Q per temperature. The observation is
two library calls — the FP64 observables pass and the charge kernel (`sck_topological_charge`) — and the measure
step (sweeps plus observation plus fold) is captured once in a CUDA graph.
"""

from __future__ import annotations

import time

import numpy as np
import torch

from . import system as sy
from .sampler import Sampler

#: Boltzmann constant in meV / K (Jex = 1 sets the energy unit)
KB = 0.086173404
PARAM_NAMES = ("Jex2", "Jex3", "Jex4", "Kan1", "KanS", "Hex", "KDM")


def build_state(params, Rd: float, L: int, angle_deg: float, shells=(1,)):
    """The nanodisk System of one parameter row [Jex2, Jex3, Jex4, Kan1, KanS, Hex, KDM] (`anneal.py:38-43`)."""
    J2, J3, J4, K1, KS, H, D = (float(v) for v in params)
    return sy.nanodot(Rd=Rd, L=L, Jex=1.0, Kan1=K1, Kan2=0.0, KanS=KS, Hex=H, KDM=D, gamma_deg=angle_deg,
                      shells=tuple(shells), J_shells={2: J2, 3: J3, 4: J4})


def active_shells(rows) -> list[int]:
    """Shells with a non-zero coupling in any state (plus shell 1): one colouring then serves every state."""
    used = {1}
    for row in rows:
        used |= {shell for shell, J in zip((2, 3, 4), row[:3]) if float(J) != 0.0}
    return sorted(used)


def check_exact(s, device="cuda", sweeps: int = 3, T: float = 0.5, seed: int = 1) -> int:
    """Spins that differ between the coloured sweep and the sequential reference chain (0 when exact)."""
    A, R = Sampler(s, 2, device, seed), Sampler(s, 2, device, seed)
    for X in (A, R):
        X.set_temperature(T)
    S1 = A.init_spins(seed=seed)
    S2 = S1.clone()
    A.sweep(S1, sweeps)
    R.reference_sweep(S2, sweeps)
    return int((S1 != S2).sum())


class Observer:
    """FP64 energy, mean magnetization vector and middle-layer charge per replica into preallocated tensors
    (graph-safe: no host work, no allocation after the first call)."""

    def __init__(self, A: Sampler):
        s = A.sys
        f64 = dict(dtype=torch.float64, device=A.device)
        self.A, self.n_act, self.mid = A, float(s.n_active), s.L3 // 2
        self.E = torch.zeros(A.B, **f64)
        self.M = torch.zeros((A.B, s.b, s.n), **f64)
        self.Q = torch.zeros(A.B, **f64)

    def __call__(self, S: torch.Tensor):
        self.A.observables(S, self.E, self.M)
        self.A.topological_charge(S, self.mid, self.Q)
        return self.E, self.M.sum(dim=1) / self.n_act, self.Q


def anneal_state(s, replicas: int, temps_K, n_therm: int, n_meas: int, every: int, seed: int, device="cuda",
                 log=print, graphs: bool | None = None):
    """Run the ladder for one state (`anneal.py:149-224`): returns obs (n_T, 8, B) = (<dE>, <dE^2>, <dM>, <dM^2>,
    <Mz>, <Q>, E_ref, M_ref), mvec (n_T, B, 3), the middle layer's s_z of replica 0 after each temperature
    (n_T, N, N), and timings. `graphs=False` launches every step from the host."""
    A = Sampler(s, replicas, device, seed)
    S = A.init_spins(seed=seed)
    observe = Observer(A)
    every = max(1, int(every))
    block = 10 * every
    nT = len(temps_K)
    obs = np.zeros((nT, 8, replicas))
    mvec = np.zeros((nT, replicas, 3), np.float32)
    snaps = np.zeros((nT, s.shape[2], s.shape[3]), np.float32)
    f64 = dict(dtype=torch.float64, device=A.device)
    E_ref, M_ref = torch.zeros(replicas, **f64), torch.zeros(replicas, **f64)
    acc = torch.zeros(6, replicas, **f64)                     # dE, dE^2, dM, dM^2, Mz, Q
    accv = torch.zeros(replicas, 3, **f64)

    def measure_step():
        A.sweep(S, every)
        E, Mv, Q = observe(S)
        dE = E - E_ref
        dM = Mv.norm(dim=1) - M_ref
        acc.add_(torch.stack([dE, dE * dE, dM, dM * dM, Mv[:, 2], Q]))
        accv.add_(Mv)

    dev = A.device
    use_graphs = dev.type == "cuda" if graphs is None else bool(graphs)
    A.set_temperature(KB * float(temps_K[0]))
    if use_graphs:
        therm = A.graph(S, block)
        with torch.cuda.device(dev):
            side = torch.cuda.Stream(device=dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                measure_step()                                # warm-up outside the capture
            torch.cuda.current_stream(dev).wait_stream(side)
            torch.cuda.synchronize(dev)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                measure_step()

        def observe_step():
            with torch.cuda.device(dev):
                g.replay()
    else:
        def therm():
            A.sweep(S, block)
        observe_step = measure_step

    t0 = time.perf_counter()
    n_obs = max(1, n_meas // every)
    for t, TK in enumerate(temps_K):
        A.set_temperature(KB * float(TK))
        for _ in range(n_therm // block):
            therm()
        if n_therm % block:
            A.sweep(S, n_therm % block)
        E, Mv, _ = observe(S)
        E_ref.copy_(E)
        M_ref.copy_(Mv.norm(dim=1))
        acc.zero_()
        accv.zero_()
        for _ in range(n_obs):
            observe_step()
        obs[t, :6] = (acc / n_obs).cpu().numpy()
        obs[t, 6] = E_ref.cpu().numpy()
        obs[t, 7] = M_ref.cpu().numpy()
        mvec[t] = (accv / n_obs).float().cpu().numpy()
        snaps[t] = S[0, 2, 0, observe.mid].float().cpu().numpy()
        if t % max(1, nT // 10) == 0 or t == nT - 1:
            log(f"    T = {TK:7.3f} K   <E>/site = {(obs[t, 6].mean() + obs[t, 0].mean()) / observe.n_act:+.4f}"
                f"   |M| = {obs[t, 7].mean() + obs[t, 2].mean():.4f}   {time.perf_counter() - t0:7.1f} s")
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    sweeps = nT * (n_therm + n_obs * every)
    return dict(obs=obs, mvec=mvec, snaps=snaps, seconds=dt, sweeps_per_chain=sweeps,
                flips_per_ns=replicas * observe.n_act * sweeps / dt / 1e9)


def reduce_obs(obs, temps, n_spins, kB: float = KB):
    """Accumulators (n_T, 8, B) -> per-temperature E, E_sd, M, M_sd, Mz, C_v, chi, Q, Q_sd (`anneal.py:227-241`)."""
    obs = np.asarray(obs)
    if obs.ndim != 3 or obs.shape[1] != 8:
        raise ValueError(f"expected (n_T, 8, batch), got {obs.shape}")
    dE, dE2, dM, dM2, Mz, Q, E_ref, M_ref = (obs[:, i] for i in range(8))
    T = np.asarray(temps)[:, None]
    E, M = dE + E_ref, dM + M_ref
    Cv = (dE2 - dE ** 2) / (kB * T ** 2 * n_spins)
    chi = (dM2 - dM ** 2) / (kB * T)
    return dict(T=np.asarray(temps), E=E.mean(1) / n_spins, E_sd=E.std(1) / n_spins, M=M.mean(1), M_sd=M.std(1),
                Mz=Mz.mean(1), Cv=Cv.mean(1), chi=chi.mean(1), Q=Q.mean(1), Q_sd=Q.std(1))

