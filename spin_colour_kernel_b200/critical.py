"""Critical-point analysis of long plain chains: the numerical core of the reference's E4 pipeline
(`src/Spin_Colour_Kernel/exp_perf.py:715-850`) on this library.

`series` runs every temperature and seed of one system size as one batch of replicas and records the FP64 energy
and the moments m^2, m^4 of the magnetization per site after every `every` sweeps (sweeps replayed from a CUDA
graph, observations from the library's observables pass). `multi_histogram` reweights all temperatures at once
(Ferrenberg-Swendsen / WHAM, in FP64), `binder_curve` turns the moments into the Binder cumulant
U = 1 - <m^4> / (3 <m^2>^2) on a temperature grid, `crossing` finds where two sizes' curves cross, and
`e4_temperatures` places a size's temperatures one canonical energy width apart around T_c.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import system as sy
from .sampler import Sampler


def e4_systems():
    """(factory, args, kwargs, dimension, 1/nu + omega) of the systems the pipeline studies."""
    return [
        (sy.ising, ("square",), {"T_ref": sy.TC["Ising square"]}, "2d", 3.0),
        (sy.ising, ("triangular",), {"T_ref": sy.TC["Ising triangular"]}, "2d", 3.0),
        (sy.ising, ("sc",), {"T_ref": sy.TC["Ising sc"]}, "3d", 2.42),
        (sy.ising, ("bcc",), {"T_ref": sy.TC["Ising bcc"]}, "3d", 2.42),
        (sy.ising, ("fcc",), {"T_ref": sy.TC["Ising fcc"]}, "3d", 2.42),
        (sy.xy, ("sc",), {"T_ref": sy.TC["XY sc"]}, "3d", 2.28),
        (sy.heisenberg, ("sc",), {"T_ref": sy.TC["Heisenberg sc"]}, "3d", 2.19),
        (sy.heisenberg, ("bcc",), {"T_ref": sy.TC["Heisenberg bcc"]}, "3d", 2.19),
    ]


def series(s: sy.System, L_box: int, temps, seeds: int, therm: int, meas: int, every: int, device="cuda",
           graphs: bool | None = None):
    """E, m^2, m^4 series (n_T, seeds, n_obs) of one size: replica r runs temperature temps[r // seeds]; sampler
    seed 12345 + L_box, initial spins from seed L_box, an observation every `every` sweeps. On a GPU the sweeps
    replay a CUDA graph (whose capture runs one warm-up sweep first, as the reference's does); `graphs=False`
    launches them from the host — the reference's CPU chain."""
    B = len(temps) * seeds
    A = Sampler(s, B, device, 12345 + L_box)
    A.set_temperature(torch.tensor(np.repeat(temps, seeds), dtype=torch.float32, device=device))
    S = A.init_spins(seed=L_box)
    k = max(1, int(every))
    use_graphs = A.device.type == "cuda" if graphs is None else bool(graphs)
    step = A.graph(S, k) if use_graphs else (lambda: A.sweep(S, k))
    for _ in range(int(math.ceil(therm / k))):
        step()
    f64 = dict(dtype=torch.float64, device=A.device)
    E_buf, M_buf = torch.zeros(B, **f64), torch.zeros((B, s.b, s.n), **f64)
    n_obs = int(math.ceil(meas / k))
    E_out, m2_out, m4_out = (torch.zeros((n_obs, B), **f64) for _ in range(3))
    N = float(s.n_active)
    for t in range(n_obs):
        step()
        A.observables(S, E_buf, M_buf)
        m = M_buf.sum(dim=1).norm(dim=1) / N
        E_out[t].copy_(E_buf)
        m2_out[t].copy_(m ** 2)
        m4_out[t].copy_(m ** 4)
    shape = (len(temps), seeds, n_obs)
    return tuple(x.T.reshape(shape).cpu().numpy() for x in (E_out, m2_out, m4_out))


def multi_histogram(E, obs, temps, grid, weights=None, device="cpu", lnZ0=None, tol=1e-10, iters=5000,
                    return_lnZ=False):
    """Canonical averages on `grid` of every observable in `obs` (each shaped like E: (temps, samples)) from the
    samples of all simulated temperatures (Ferrenberg and Swendsen, PRL 63, 1195 (1989)). The free energies
    ln Z_k solve the self-consistent equations
        ln Z_k = ln sum_samples w exp(-beta_k E) / sum_j N_j exp(-beta_j E - ln Z_j),   ln Z_0 = 0,
    iterated from thermodynamic integration until they move by less than `tol`; `weights` are per-sample
    multiplicities (bootstrap), energies are shifted by their mean so exponents stay small. FP64 throughout."""
    f64 = torch.float64
    En = torch.as_tensor(np.asarray(E, np.float64), dtype=f64, device=device)
    nT = En.shape[0]
    w = torch.ones_like(En) if weights is None else torch.as_tensor(np.asarray(weights, np.float64), dtype=f64,
                                                                    device=device)
    beta = 1.0 / torch.as_tensor(np.asarray(temps, np.float64), dtype=f64, device=device)
    shift = float((En * w).sum() / w.sum())
    x = (En - shift).reshape(-1)
    log_w = torch.log(w.reshape(-1))
    log_n = torch.log(w.sum(dim=1))
    if lnZ0 is None:
        mean_e = (En * w).sum(dim=1) / w.sum(dim=1) - shift
        lnZ = torch.zeros(nT, dtype=f64, device=device)
        lnZ[1:] = torch.cumsum(-0.5 * (beta[1:] - beta[:-1]) * (mean_e[1:] + mean_e[:-1]), 0)
    else:
        lnZ = torch.as_tensor(np.asarray(lnZ0, np.float64), dtype=f64, device=device).clone()
    bx = beta[:, None] * x[None, :]
    for _ in range(int(iters)):
        denom = torch.logsumexp(log_n[:, None] - bx - lnZ[:, None], dim=0)
        nxt = torch.logsumexp(log_w[None, :] - bx - denom[None, :], dim=1)
        nxt = nxt - nxt[0]
        converged = float((nxt - lnZ).abs().max()) < tol
        lnZ = nxt
        if converged:
            break
    denom = torch.logsumexp(log_n[:, None] - bx - lnZ[:, None], dim=0)
    g = 1.0 / torch.as_tensor(np.asarray(grid, np.float64), dtype=f64, device=device)
    prob = torch.softmax(log_w[None, :] - g[:, None] * x[None, :] - denom[None, :], dim=1)
    out = [(prob @ torch.as_tensor(np.asarray(o, np.float64), dtype=f64, device=device).reshape(-1)).cpu().numpy()
           for o in obs]
    return (out, lnZ.cpu().numpy()) if return_lnZ else out


def e4_temperatures(Tc: float, sigma_E: float, ntemps: int, window: float) -> np.ndarray:
    """ntemps temperatures around Tc, neighbours one canonical energy width apart (delta T / T = T / sigma_E),
    never more than +-window relative."""
    half = min(window, 0.5 * (ntemps - 1) * Tc / sigma_E)
    return Tc * (1 + np.linspace(-half, half, ntemps))


def binder_curve(E, m2, m4, temps, grid, weights=None, device="cpu", lnZ0=None):
    """Binder cumulant U = 1 - <m^4> / (3 <m^2>^2) on `grid`, reweighted from every temperature; returns (U, lnZ)."""
    nT = len(temps)
    (a2, a4), lnZ = multi_histogram(np.reshape(E, (nT, -1)), [np.reshape(m2, (nT, -1)), np.reshape(m4, (nT, -1))],
                                    temps, grid, device=device, lnZ0=lnZ0, return_lnZ=True,
                                    weights=None if weights is None else np.reshape(weights, (nT, -1)))
    return 1.0 - a4 / (3.0 * a2 * a2), lnZ


def crossing(grid, u1, u2) -> float:
    """Temperature where two curves cross (linear interpolation at the middle sign change), NaN if none."""
    d = np.asarray(u1) - np.asarray(u2)
    flips = np.flatnonzero(np.sign(d[:-1]) != np.sign(d[1:]))
    if flips.size == 0:
        return float("nan")
    j = flips[flips.size // 2]
    return float(grid[j] - d[j] * (grid[j + 1] - grid[j]) / (d[j + 1] - d[j]))
