"""The one-state ladder runner on the GPU against the reference's own runner.

`tests/golden/simulate.npz` holds the outputs of the reference's `simulate_state` on its CPU path
(`make_golden.py simulate`) for two Ising systems, whose chains are bit-exact on every backend: the runner
here, without graphs (the reference's CPU path captures none), must return the same energies, moments,
magnetizations and configurations. With graphs the chain gains the warm-up sweeps of the captures (as the
reference's GPU path does); that run is checked for its shapes and invariants, and the fused device fold of one
observation against the same fold done in torch.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden" / "simulate.npz"

# the systems of make_golden.py:_simulate (the reference's build_system for these states)
RUNS = {
    "square": (lambda: sy.System("ising square", 1, cr.make("square", (1,)), (8, 8), (True, True), {1: 1.0},
                                 h=(0.1,)),
               dict(replicas=4, temps=[3.0, 2.5, 2.0], n_therm=4, n_meas=6, every=2, config_every=2, seed=1)),
    "sc_word": (lambda: sy.System("ising sc", 1, cr.make("sc", (1,)), (4, 4, 4), (True, True, True), {1: 1.0}),
                dict(replicas=32, temps=[5.0, 4.0], n_therm=3, n_meas=4, every=1, config_every=1, seed=2)),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200 import build
    build.build()


@pytest.mark.parametrize("key", sorted(RUNS))
def test_ladder_runner_matches_reference_runner(key):
    from spin_colour_kernel_b200.simulate import simulate_state
    gold = np.load(GOLD)
    build, kw = RUNS[key]
    r = simulate_state(build(), device="cuda", kB=1.0, log=lambda m: None, graphs=False, **kw)
    for f in ("E", "E2", "Mabs", "M2"):
        np.testing.assert_allclose(r[f], gold[f"{key}_{f}"], rtol=1e-12, atol=1e-9, err_msg=f)
    np.testing.assert_allclose(r["M"], gold[f"{key}_M"], rtol=0, atol=1e-7)
    assert np.array_equal(r["configs"], gold[f"{key}_configs"])
    assert np.array_equal(r["config_temperatures"], gold[f"{key}_config_temperatures"])


def test_ladder_runner_with_graphs_keeps_shapes_and_invariants():
    from spin_colour_kernel_b200.simulate import simulate_state, temperature_ladder
    s = sy.System("xy square", 2, cr.make("square", (1,)), (6, 6), (True, True), {1: 1.0}, h=(0.1, 0.0))
    temps = temperature_ladder(2.0, 1.0, 0.5)
    r = simulate_state(s, replicas=3, temps=temps, n_therm=4, n_meas=4, every=2, config_every=2, seed=1,
                       device="cuda", kB=1.0, log=lambda m: None)
    nT = len(temps)
    assert r["M"].shape == (3, nT, 3) and r["E"].shape == (3, nT) and r["E2"].shape == (3, nT)
    assert r["Mabs"].shape == (3, nT) and r["M2"].shape == (3, nT)
    assert r["configs"].shape == (3, 2, 36, 3) and list(r["config_temperatures"]) == [2.0, 1.0]
    assert np.allclose(np.linalg.norm(r["configs"], axis=-1), 1.0, atol=1e-5)
    assert np.all(r["configs"][..., 2] == 0)
    assert np.all(r["Mabs"] <= 1 + 1e-6) and np.all(r["E2"] >= r["E"] ** 2 - 1e-6)


@pytest.mark.parametrize("build", [lambda: sy.heisenberg("bcc", 6), lambda: sy.xy("triangular", 12),
                                   lambda: sy.ising("sc", 6)])
def test_device_fold_equals_torch_fold(build):
    """Two observations folded on the device against the same fold written in torch from sck_observables."""
    from spin_colour_kernel_b200.sampler import Sampler
    s = build()
    B = 5
    A = Sampler(s, B, device="cuda", seed=4)
    A.set_temperature(torch.linspace(0.5, 3.0, B))
    S = A.init_spins(seed=9)
    f64 = dict(dtype=torch.float64, device="cuda")
    E_ref = A.observables(S)[0] + 0.25
    acc, accv = torch.zeros((4, B), **f64), torch.zeros((B, s.n), **f64)
    E, M = torch.zeros(B, **f64), torch.zeros((B, s.b, s.n), **f64)
    want, wantv = torch.zeros_like(acc), torch.zeros_like(accv)
    for _ in range(2):
        A.sweep(S, 1)
        A.observe(S, E_ref, acc, accv, E, M)
        E2, M2 = A.observables(S)
        mv = M2.sum(dim=1) / float(s.n_active)
        d = E2 - E_ref
        a = mv.norm(dim=1)
        want += torch.stack([d, d * d, a, a * a])
        wantv += mv
        assert torch.equal(E, E2) and torch.equal(M, M2)
    torch.testing.assert_close(acc, want, rtol=1e-14, atol=1e-12)
    torch.testing.assert_close(accv, wantv, rtol=1e-14, atol=1e-15)
