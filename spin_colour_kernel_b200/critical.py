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


# ------------------------------------------------------------------------------------------ multi-size driver
def holm(p) -> list[float]:
    """Holm's step-down adjustment of a family of p-values (each p times the number of hypotheses not yet
    rejected, made monotone, capped at 1)."""
    p = np.asarray(p, np.float64)
    adj = np.zeros(p.size)
    running = 0.0
    for rank, i in enumerate(np.argsort(p)):
        running = max(running, (p.size - rank) * p[i])
        adj[i] = min(1.0, running)
    return adj.tolist()


def probe_tau(s: sy.System, L_box: int, Tc: float, seeds: int, device="cuda", start: int = 2000,
              cap: int = 100_000, ratio: int = 50):
    """tau_int of m^2 at Tc from probes of growing length (x4 from `start`, at most `cap`) until the probe reaches
    `ratio` tau: (tau, probe length, whether it reached ratio tau, energy spread of one configuration)."""
    from .stats import integrated_tau
    length = int(start)
    while True:
        E, m2, _ = series(s, L_box, [Tc], seeds, max(500, length // 4), length, 1, device)
        tau = integrated_tau(m2[0].T)
        if length >= ratio * tau or length >= cap:
            return tau, length, bool(length >= ratio * tau), float(E[0].std(axis=1).mean())
        length = min(cap, 4 * length)


def _size_box(s0: sy.System, L: int) -> int:
    """Box side of size L: triangular boxes take the nearest multiple of 3 (a 3-colouring of the periodic box)."""
    return 3 * int(round(L / 3)) if s0.crystal.name == "triangular" else L


def _make(maker, args, L, kw, acceptance):
    s = maker(*args, L, **kw)
    if acceptance != s.acceptance:
        s = sy.System(s.name, s.n, s.crystal, s.box, s.periodic, s.J, T_ref=s.T_ref, acceptance=acceptance)
    return s


def crossing_estimate(data: dict, x: float, weights=None, device="cpu", lnZ_cache=None, points: int = 241):
    """T_c from Binder crossings of consecutive sizes: for each pair (L1, L2), both curves reweighted onto the
    temperatures both sizes cover, crossed; with two or more crossings, the intercept of a straight-line fit of
    T_cross against sqrt(L1 L2)^-x, else the last crossing. `weights` are per-seed multiplicities (bootstrap);
    `lnZ_cache` keeps each size's free energies from the unweighted pass as the next passes' starting point.
    Returns (estimate, [(sqrt(L1 L2), T_cross)], {(L1, L2): (grid, U1, U2)})."""
    Ls = sorted(data)
    curves, cross = {}, []
    for a, b in zip(Ls[:-1], Ls[1:]):
        grid = np.linspace(max(data[a]["temps"][0], data[b]["temps"][0]),
                           min(data[a]["temps"][-1], data[b]["temps"][-1]), points)
        us = []
        for L in (a, b):
            d = data[L]
            w = None if weights is None else np.broadcast_to(weights[None, :, None], d["E"].shape)
            u, lnZ = binder_curve(d["E"], d["m2"], d["m4"], d["temps"], grid, weights=w, device=device,
                                  lnZ0=None if lnZ_cache is None else lnZ_cache.get(L))
            if lnZ_cache is not None and weights is None:
                lnZ_cache[L] = lnZ
            us.append(u)
        curves[(a, b)] = (grid, us[0], us[1])
        t = crossing(grid, us[0], us[1])
        if np.isfinite(t):
            cross.append((math.sqrt(a * b), t))
    if len(cross) >= 2:
        X = np.array([l ** (-x) for l, _ in cross])
        Y = np.array([t for _, t in cross])
        return float(np.polyfit(X, Y, 1)[1]), cross, curves
    return (cross[-1][1] if cross else float("nan")), cross, curves


def e4(out, device="cuda", sizes2d=(32, 64, 128, 256), sizes3d=(16, 24, 32, 48), seeds: int = 10,
       window: float = 0.03, ntemps: int = 9, meas: int = 20000, boots: int = 2000, only=None, tag: str = "E4",
       probe_cap: int = 100_000, acceptance: str = "metropolis", probe_start: int = 2000, log=print):
    """The multi-size critical-point study (the reference's E4, `exp_perf.py:846-950`) on this library: for each
    system of `e4_systems()` (or those named in `only`) and each size, tau_int at T_c from a growing probe,
    `ntemps` temperatures one energy width apart (within +-window), thermalisation of max(1000, 20 tau) sweeps,
    an observation every max(1, tau / 2, meas / 2000) sweeps, the raw series saved to
    `<out>/<tag>-<system>-L<L>.npz`; then T_c from Binder crossings of consecutive sizes extrapolated in
    L^-(1/nu + omega), a bootstrap over seeds (95 % interval, two-sided p-value of the reference T_c), Holm's
    adjustment across systems and a verdict (supported / not supported / inconclusive when the half-width
    exceeds 0.5 % of T_c). Writes and returns `<out>/<tag>.json`'s payload."""
    import json
    import time
    from pathlib import Path
    from .stats import integrated_tau
    out = Path(out)
    out.mkdir(parents=True, exist_ok=True)
    rdev = device if str(device).startswith("cuda") and torch.cuda.is_available() else "cpu"
    rows = []
    for maker, args, kw, dim, x in e4_systems():
        probe = _make(maker, args, 6 if args[0] == "triangular" else 4, kw, acceptance)
        if only and probe.name not in only:
            continue
        Tc = kw["T_ref"]
        t0 = time.time()
        data = {}
        for L in (sizes2d if dim == "2d" else sizes3d):
            Lb = _size_box(probe, L)
            s = _make(maker, args, Lb, kw, acceptance)
            tau, P, resolved, sigma_E = probe_tau(s, Lb, Tc, seeds, device, start=probe_start, cap=probe_cap)
            temps = e4_temperatures(Tc, sigma_E, ntemps, window)
            therm = int(max(1000, 20 * tau))
            every = max(1, int(round(tau / 2)), meas // 2000)
            E, m2, m4 = series(s, Lb, temps, seeds, therm, meas, every, device)
            mid = int(np.argmin(np.abs(temps - Tc)))
            tau_prod = every * integrated_tau(m2[mid].T)
            np.savez_compressed(out / f"{tag}-{probe.name.replace(' ', '_')}-L{Lb}.npz", E=E,
                                m2=m2.astype(np.float32), m4=m4.astype(np.float32), temps=temps, tau=tau,
                                therm=therm, every=every)
            data[Lb] = {"E": E, "m2": m2, "m4": m4, "temps": temps, "tau": tau, "probe_sweeps": P,
                        "tau_resolved": resolved, "sigma_E": sigma_E, "therm": therm, "every": every,
                        "tau_production": tau_prod, "therm_over_tau_production": therm / tau_prod}
            log(f"E4 {probe.name:20s} L={Lb} tau={tau:.1f} (probe {P}, resolved {resolved}) tau_prod={tau_prod:.1f} "
                f"therm={therm} every={every} window=+-{(temps[-1] / Tc - 1):.4%} {time.time() - t0:.0f}s")
        lnZ = {}
        est, pairs, curves = crossing_estimate(data, x, device=rdev, lnZ_cache=lnZ)
        rng = np.random.default_rng(1)
        bs = np.array([crossing_estimate(data, x, weights=np.bincount(rng.integers(0, seeds, seeds),
                                                                      minlength=seeds).astype(np.float64),
                                         device=rdev, lnZ_cache=lnZ)[0] for _ in range(boots)])
        bs = bs[np.isfinite(bs)]
        lo, hi = np.quantile(bs, [0.025, 0.975]) if bs.size > 10 else (np.nan, np.nan)
        half = (hi - lo) / 2 / Tc
        p = float(min(1.0, 2 * min(np.mean(bs <= Tc), np.mean(bs >= Tc)))) if bs.size else float("nan")
        keys = ("tau", "probe_sweeps", "tau_resolved", "sigma_E", "therm", "every", "tau_production",
                "therm_over_tau_production")
        Ls = sorted(data)
        rows.append({"system": probe.name, "T_ref": Tc, "estimate": est, "low": float(lo), "high": float(hi),
                     "half_width_over_Tc": float(half), "p_reference": p, "pair_crossings": pairs, "sizes": Ls,
                     "temps": {L: data[L]["temps"].tolist() for L in Ls}, "correction_exponent": x,
                     "reweighting": "multi-histogram", "declared": {L: {k: data[L][k] for k in keys} for L in Ls},
                     "binder": {f"{a}-{b}": {"grid": g.tolist(), str(a): ua.tolist(), str(b): ub.tolist()}
                                for (a, b), (g, ua, ub) in curves.items()},
                     "seconds": time.time() - t0})
        log(f"E4 {probe.name:20s} Tc={est:.5f} [{lo:.5f},{hi:.5f}] ref {Tc:.5f} half {half:.4%}")
    for r, pa in zip(rows, holm([r["p_reference"] if np.isfinite(r["p_reference"]) else 1.0 for r in rows])):
        r["p_holm"] = pa
        r["verdict"] = ("inconclusive" if not (r["half_width_over_Tc"] <= 0.005) else
                        ("supported" if pa >= 0.05 else "not supported"))
    payload = {"experiment": tag, "rows": rows,
               "params": {"sizes2d": list(sizes2d), "sizes3d": list(sizes3d), "seeds": seeds, "window": window,
                          "ntemps": ntemps, "meas": meas, "boots": boots, "probe_cap": probe_cap,
                          "reweighting": "multi-histogram"}}
    (out / f"{tag}.json").write_text(json.dumps(payload, indent=2, default=float))
    return payload
