"""Pin the CPU oracle against the reference's own outputs (tests/golden, made by tests/golden/make_golden.py).

Every fixture was produced by the reference's CPU path (the Triton interpreter). The oracle must reproduce the
spins bit for bit after every recorded sweep, for every system and mode, and the FP64 energies and
magnetizations to rounding.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import cases as C
from oracle import bitwise as obw
from oracle import observables as obs
from oracle import philox
from oracle import sweep as osw
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

GOLD = Path(__file__).resolve().parent / "golden"
FAST = [k for k in C.CASES if (GOLD / f"{k}.npz").exists() and not C.CASES[k].get("bitwise")
        and C.CASES[k]["sweeps"] <= 10]
BITWISE = [k for k in C.CASES if (GOLD / f"{k}.npz").exists() and C.CASES[k].get("bitwise")]


def load(name):
    return dict(np.load(GOLD / f"{name}.npz"))


def beta_of(T):
    return (np.float32(1.0) / np.asarray(T, np.float32)).astype(np.float32)


def storage(case, sys_, S0):
    if sys_.n == 1:
        return S0.astype(np.int8)
    return S0.astype(np.float32)


@pytest.mark.parametrize("name", FAST)
def test_oracle_reproduces_reference_chain(name):
    case = C.CASES[name]
    g = load(name)
    s = case["build"](sy, cr)
    assert s.colouring.n_colours == int(g["n_colours"])
    assert [tuple(c) for c in g["classes"]] == osw.classes(s)
    S = storage(case, s, g["S0"]).copy()
    beta = beta_of(g["T"])
    state = [case["seed"], 0]
    snaps = {int(k): i for i, k in enumerate(g["snap_ids"])}
    for k in range(1, case["sweeps"] + 1):
        osw.sweep(s, S, beta, state)
        if k in snaps:
            ref = g["snaps"][snaps[k]]
            assert np.array_equal(S, ref.astype(S.dtype)), f"{name}: sweep {k}: {(S != ref).sum()} spins differ"
        np.testing.assert_allclose(obs.energy(s, S), g["E"][k - 1], rtol=1e-10, atol=1e-9)
        np.testing.assert_allclose(obs.magnetization(S), g["M"][k - 1], rtol=1e-10, atol=1e-9)


@pytest.mark.slow
def test_oracle_reproduces_reference_workload1_200_sweeps():
    """2D Ising square L=32, 32 replicas at T in {1.5, 2.0, 2.269, 3.0}, key 1234, init seed 0, 200 sweeps:
    per-sweep energies of all replicas and spins at sweeps 1, 2, 10, 50, 100, 200."""
    name = "w1_ising_square32"
    if not (GOLD / f"{name}.npz").exists():
        pytest.skip("fixture not generated")
    case = C.CASES[name]
    g = load(name)
    s = case["build"](sy, cr)
    S = g["S0"].astype(np.int8).copy()
    beta = beta_of(g["T"])
    state = [case["seed"], 0]
    snaps = {int(k): i for i, k in enumerate(g["snap_ids"])}
    for k in range(1, case["sweeps"] + 1):
        osw.sweep(s, S, beta, state)
        if k in snaps:
            assert np.array_equal(S, g["snaps"][snaps[k]]), f"sweep {k}"
        np.testing.assert_allclose(obs.energy(s, S), g["E"][k - 1], rtol=0, atol=1e-9)


@pytest.mark.parametrize("name", BITWISE)
def test_bitwise_oracle_reproduces_reference_kernel(name):
    case = C.CASES[name]
    g = load(name)
    s = case["build"](sy, cr)
    beta = beta_of(g["T"])
    W = -(-case["B"] // 32)
    table = obw.p_fixed(s, beta.reshape(W, 32)[:, 0]) if case.get("independent") else \
        obw.p_table(s, beta.reshape(W, 32)[:, 0])
    assert np.array_equal(table, g["ptab"])
    x = g["S0"][:, 0].astype(np.int64)
    for k in range(1, case["sweeps"] + 1):
        x = obw.sweep(s, x, table, case["seed"], k - 1, independent=bool(case.get("independent")))
        assert np.array_equal(x, g["snaps"][k - 1][:, 0]), f"{name}: sweep {k}"


def test_philox_matches_triton():
    g = load("philox")
    N = int(g["N"])
    for i, sd in enumerate(g["seeds"]):
        off = np.arange(N, dtype=np.int64) * int(g["offset_mul"]) + int(g["offset_add"])
        assert np.array_equal(philox.uniform4(int(sd), philox.int32_counter(off)), g["rand4x"][i])
        offi = np.arange(N, dtype=np.int64) * int(g["int_mul"]) + int(g["int_add"])
        assert np.array_equal(philox.raw4(int(sd), philox.int32_counter(offi)), g["randint4x"][i])
    for j, b in enumerate((0, 1, 1234, 99991)):
        assert [philox.sweep_seed(b, t) for t in range(50)] == list(g["sweep_seeds"][j])


def test_acceptance_tables_match_reference():
    g = load("tables")
    betas = g["betas"]
    systems = {"square": sy.ising("square", 4), "sc": sy.ising("sc", 4), "fcc": sy.ising("fcc", 4),
               "triangular": sy.ising("triangular", 6)}
    for key, s in systems.items():
        for acc in ("metropolis", "barker"):
            s.acceptance = acc
            assert np.array_equal(obw.p_table(s, betas), g[f"{key}_{acc}_p"])
            assert np.array_equal(obw.p_fixed(s, betas), g[f"{key}_{acc}_P"])
