"""Long-run statistics of the vector models: the GPU chain against the oracle's chain.

Over thousands of sweeps XY and Heisenberg chains of the GPU and of the oracle (its C port, the reference's
arithmetic with the C library's transcendental functions) part ways after a decision whose uniform falls within
rounding of its acceptance probability flips. Both must still sample the same distribution: per temperature, the
mean energy per site, |m|, the specific heat and the susceptibility of the two chains must agree within 2 sigma.
The estimators follow the reference's run collector (Spin_Colour_Kernel/simulate.py:511-527): per replica the
time averages of E, E^2, |m| and |m|^2 give Cv = var(E) / (T^2 N) and chi = N var(|m|) / T; a temperature's value
is the mean over its replicas (independent chains), its sigma the standard error of that mean.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import cases as C
from oracle import native
from oracle import observables as obs
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

pytestmark = pytest.mark.gpu

SWEEPS, THERM, EVERY = 2000, 400, 2


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200 import build
    build.build()
    native.build()


def _estimates(E, M, T, N):
    """E (samples, B) total energies, M (samples, B, n) magnetization vectors; per-replica estimators, then
    mean and standard error over the replicas of each temperature."""
    m = np.linalg.norm(M, axis=2) / N
    per = {"e": E.mean(0) / N, "absm": m.mean(0),
           "Cv": np.maximum((E ** 2).mean(0) - E.mean(0) ** 2, 0.0) / (T ** 2 * N),
           "chi": N * np.maximum((m ** 2).mean(0) - m.mean(0) ** 2, 0.0) / T}
    out = {}
    for t in np.unique(T):
        sel = T == t
        out[float(t)] = {k: (v[sel].mean(), v[sel].std(ddof=1) / np.sqrt(sel.sum())) for k, v in per.items()}
    return out


@pytest.mark.parametrize("model", ["heisenberg-bcc-j1j2-quad", "xy-square-field"])
def test_long_run_observables_agree_with_oracle_chain_within_2_sigma(model):
    from spin_colour_kernel_b200.sampler import Sampler
    if model.startswith("heisenberg"):
        s = C.heisenberg_bcc_j1j2(sy, cr, 8)                  # 1,024 sites
        temps, layout = (1.2, 2.4), "quad"
    else:
        s = C.xy_periodic_field(sy, cr, "square", 32)         # 1,024 sites
        temps, layout = (0.7, 1.2), "reference"
    B = 64
    T = np.repeat(np.asarray(temps, np.float32), B // len(temps))
    A = Sampler(s, B, device="cuda", seed=41, layout=layout)
    A.set_temperature(torch.from_numpy(T))
    S = A.init_spins(seed=6)
    x = A.unpack(S).cpu().numpy()
    beta = (np.float32(1.0) / T).astype(np.float32)
    state = [41, 0]
    N = s.n_active
    Eg, Mg, Eo, Mo = [], [], [], []
    for k in range(SWEEPS // EVERY):
        A.sweep(S, EVERY)
        x = native.sweep(s, x, beta, state, EVERY)
        if (k + 1) * EVERY > THERM:
            E, M = A.observables(S)
            Eg.append(E.cpu().numpy())
            Mg.append(M.sum(dim=1).cpu().numpy())
            Eo.append(obs.energy(s, x))
            Mo.append(obs.magnetization(x).sum(axis=1))
    g = _estimates(np.asarray(Eg), np.asarray(Mg), T, N)
    o = _estimates(np.asarray(Eo), np.asarray(Mo), T, N)
    worst = 0.0
    for t in g:
        for key in ("e", "absm", "Cv", "chi"):
            (a, sa), (b, sb) = g[t][key], o[t][key]
            z = abs(a - b) / max(np.hypot(sa, sb), 1e-300)
            print(f"{model} T={t:.2f} {key}: gpu {a:.6g} +- {sa:.2g}, oracle {b:.6g} +- {sb:.2g}, z = {z:.2f}")
            worst = max(worst, z)
            assert z <= 2.0, f"{model} T={t}: {key} differs by {z:.2f} sigma"
    print(f"{model}: largest deviation {worst:.2f} sigma")
