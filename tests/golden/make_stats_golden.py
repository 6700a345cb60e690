"""Golden values of the reference's chain statistics (integrated_tau, boot_ci) on seeded AR(1) series.

Run in a container that holds the reference sources:
    python tests/golden/make_stats_golden.py [--ref /root/reference/src]
Writes tests/golden/stats.npz.
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np


def series():
    rng = np.random.default_rng(11)
    out = []
    for n, chains, phi in [(1, 1, 0.0), (2, 3, 0.5), (64, 1, 0.0), (500, 4, 0.9), (1500, 2, 0.97), (300, 2, -0.6),
                           (400, 6, 0.5), (50, 3, 0.999)]:
        x = np.zeros((n, chains))
        e = rng.normal(size=(n, chains))
        for t in range(n):
            x[t] = (phi * x[t - 1] if t else 0.0) + e[t]
        out.append(x)
    out.append(np.ones((40, 2)))                           # constant: tau 1
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference/src")
    args = ap.parse_args()
    sys.path.insert(0, args.ref)
    from Spin_Colour_Kernel import exp_core, exp_perf
    data = {}
    for i, x in enumerate(series()):
        data[f"x{i}"] = x
        data[f"tau{i}"] = np.array([exp_core.integrated_tau(x), exp_core.integrated_tau(x, c=4.0)])
        data[f"ci{i}"] = np.array(exp_perf.boot_ci(x[:, 0], n=300, seed=i))
    np.savez_compressed(Path(__file__).with_name("stats.npz"), **data)


if __name__ == "__main__":
    main()
