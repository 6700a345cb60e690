"""Chain statistics against the reference's own integrated_tau and boot_ci (tests/golden/stats.npz, made by
tests/golden/make_stats_golden.py from the reference)."""

from __future__ import annotations

from pathlib import Path

import numpy as np

from spin_colour_kernel_b200 import stats

GOLD = np.load(Path(__file__).parent / "golden" / "stats.npz")


def test_integrated_tau_matches_reference():
    n = len([k for k in GOLD.files if k.startswith("x")])
    assert n >= 8
    for i in range(n):
        x = GOLD[f"x{i}"]
        want = GOLD[f"tau{i}"]
        np.testing.assert_allclose([stats.integrated_tau(x), stats.integrated_tau(x, c=4.0)], want, rtol=1e-12,
                                   atol=1e-12, err_msg=f"series {i} {x.shape}")


def test_boot_ci_matches_reference():
    for i in range(len([k for k in GOLD.files if k.startswith("ci")])):
        x = GOLD[f"x{i}"][:, 0]
        np.testing.assert_allclose(stats.boot_ci(x, n=300, seed=i), GOLD[f"ci{i}"], rtol=1e-12, atol=1e-12)


def test_tau_of_ar1_is_close_to_its_closed_form():
    rng = np.random.default_rng(0)
    phi, n, chains = 0.8, 20000, 4
    x = np.zeros((n, chains))
    e = rng.normal(size=(n, chains))
    for t in range(1, n):
        x[t] = phi * x[t - 1] + e[t]
    assert abs(stats.integrated_tau(x) - (1 + phi) / (1 - phi)) < 0.6
