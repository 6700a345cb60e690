"""The C port of the oracle (oracle/cpu_sweep.c) against the reference's recorded chains, on the CPU.

The port is the timed CPU baseline of bench.py (its `cpu_baseline` leg and the `--impl reference` arm), so it
must compute the reference's chain: Ising bit-exact on every plain fixture (per-sweep energies and
magnetizations too where the fixture records them every sweep: all 200 sweeps of the 2D Ising workload), XY and
Heisenberg within the vector-model tolerance (per-spin |delta| <= 1e-5, the fraction of spins beyond it
reported and bounded). Packed fixtures hold the int8 chain (the reference's packed path equals it).
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import cases as C
from oracle import native
from oracle import observables as obs
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

GOLD = Path(__file__).resolve().parent / "golden"
VEC_TOL = 1e-5
PLAIN = [k for k in C.CASES if (GOLD / f"{k}.npz").exists() and not C.CASES[k].get("bitwise")]


@pytest.fixture(scope="module", autouse=True)
def _built():
    native.build()
    if not native.available():
        pytest.fail("the oracle's C port did not build")


@pytest.mark.parametrize("name", PLAIN)
def test_c_port_matches_reference_fixture(name):
    case = C.CASES[name]
    g = dict(np.load(GOLD / f"{name}.npz"))
    s = case["build"](sy, cr)
    x = g["S0"].astype(np.float32)
    beta = (np.float32(1.0) / g["T"].astype(np.float32)).astype(np.float32)
    state = [int(case["seed"]), 0]
    snaps = {int(k): i for i, k in enumerate(g["snap_ids"])}
    every_sweep = g["E"].shape[0] == case["sweeps"]
    fracs = []
    for k in range(1, case["sweeps"] + 1):
        x = native.sweep(s, x, beta, state, 1, nthreads=2)
        if k in snaps:
            ref = g["snaps"][snaps[k]]
            if s.n == 1:
                diff = int((x.astype(np.int8) != ref).sum())
                assert diff == 0, f"{name}: sweep {k}: {diff} Ising spins differ"
            else:
                d = np.abs(x.astype(np.float64) - ref.astype(np.float64))
                frac = float((d > VEC_TOL).any(axis=1).mean())
                fracs.append(frac)
                assert frac <= 0.02, f"{name}: sweep {k}: {frac:.4f} of spins beyond {VEC_TOL}"
        if s.n == 1 and every_sweep:
            np.testing.assert_allclose(obs.energy(s, x), g["E"][k - 1], rtol=1e-12, atol=1e-9,
                                       err_msg=f"{name}: energy after sweep {k}")
            np.testing.assert_allclose(obs.magnetization(x), g["M"][k - 1], rtol=1e-12, atol=1e-9,
                                       err_msg=f"{name}: magnetization after sweep {k}")
    assert state[1] == case["sweeps"]
    if fracs:
        print(f"{name}: fraction of spins beyond {VEC_TOL} per recorded sweep: {fracs}")


def test_c_port_covers_the_workload_fixtures():
    for need in ("w1_ising_square32", "w3_heis_bcc4_j1j2", "heis_bcc2", "w5_ising_sc8", "ising_sc_j1j2_field",
                 "ising_masked_field_barker", "nanodot_small"):
        assert need in PLAIN, need


def test_c_port_ising_exp_table_covers_open_masked_boxes():
    """Every argument an open, masked, J1-J2 Ising chain reaches is in the enumerated table (the port raises on a
    miss), over several sweeps at several temperatures."""
    s = sy.System("Ising sc J1-J2 open masked", 1, cr.make("sc", (1, 2)), (5, 4, 3), (False, True, False),
                  {1: 1.0, 2: -0.35}, h=(0.2,), mask=np.random.default_rng(1).random((1, 3, 4, 5)) > 0.2)
    rng = np.random.default_rng(2)
    x = (rng.integers(0, 2, (6, 1) + s.shape) * 2 - 1).astype(np.float32) * s.site_mask()
    beta = (np.float32(1.0) / np.linspace(0.5, 5.0, 6).astype(np.float32)).astype(np.float32)
    native.sweep(s, x, beta, [3, 0], 5, nthreads=2)


BITWISE = [k for k in C.CASES if (GOLD / f"{k}.npz").exists() and C.CASES[k].get("bitwise")]


@pytest.mark.parametrize("name", BITWISE)
def test_c_port_bitwise_matches_reference_fixture(name):
    """The port's bitwise chain (shared and independent draws) against the reference's recorded chains with the
    reference's own tables, spin for spin after every sweep."""
    case = C.CASES[name]
    g = dict(np.load(GOLD / f"{name}.npz"))
    s = case["build"](sy, cr)
    x = g["S0"][:, 0]
    for k in range(1, case["sweeps"] + 1):
        x = native.bitwise_sweep(s, x, g["ptab"], int(case["seed"]), k - 1, 1,
                                 independent=bool(case.get("independent")), nthreads=2)
        assert np.array_equal(x, g["snaps"][k - 1][:, 0]), f"{name}: sweep {k}"


def test_c_port_bitwise_equals_numpy_oracle_on_chosen_words():
    """Global word indices enter the counters: words 3 and 6 of a larger batch, run on their own, equal the NumPy
    oracle's restatement for both draw modes, over several sweeps."""
    from oracle import bitwise as obw
    s = sy.ising("sc", 6)
    rng = np.random.default_rng(4)
    x0 = (rng.integers(0, 2, (64,) + s.shape) * 2 - 1).astype(np.int8)
    beta = np.array([0.2, 0.35])
    for independent in (False, True):
        tab = obw.p_fixed(s, beta) if independent else obw.p_table(s, beta)
        a = native.bitwise_sweep(s, x0, tab, 7, 0, 3, independent=independent, words=[3, 6], nthreads=2)
        b = x0.astype(np.int64)
        for k in range(3):
            b = obw.sweep(s, b, tab, 7, k, independent=independent, words=[3, 6])
        assert np.array_equal(a, b.astype(np.int8)), independent
