"""The named workloads of the benchmark, as seeded synthetic inputs (no datasets; every input is reproducible).

  ising_square_32        2D Ising square L=32, periodic, J=1, h=0; 32 replicas = 8 per T in {1.5, 2.0, 2.269, 3.0};
                         int8 spins from seed 0; Philox key 1234.
  ising_sc_128_bitwise   3D Ising sc L=128, periodic, J=1; 1024 replicas as two counter-legal instances of 512
                         (1024 x 128^3 reaches the int32 Philox counter limit), 16 T linear in [4.0, 5.0], two
                         words (64 replicas) per T; hot start from seed 1.
  heisenberg_bcc_64      3D Heisenberg bcc 64^3 cells, periodic, J1=1, J2=0.3, cubic K1=0.05, h=0.1 z; 64 replicas x
                         24 T linear in [0.5, 2.5]; unit vectors uniform on the sphere from seed 2.
  xy_ragged_96           96 XY systems: 48 square + 48 triangular, L log-uniform in [16, 512] (seed 3), alternately
                         periodic and circular nanodisk masks of radius 0.45 L in an open box; J1=1, h=(0.05, 0);
                         32 replicas each at one T ~ U[0.6, 1.2]; angles uniform in [0, 2 pi) -> (cos, sin). A
                         periodic box without a seam-compatible colouring falls back to open boundaries, as the
                         reference's run driver does (Spin_Colour_Kernel/simulate.py:234-240).
"""

from __future__ import annotations

import numpy as np

from . import crystals as cr
from . import system as sy


def heisenberg_bcc(L: int = 64) -> sy.System:
    c = cr.make("bcc", (1, 2))
    return sy.System("Heisenberg bcc J1-J2", 3, c, (L, L, L), (True,) * 3, {1: 1.0, 2: 0.3}, h=(0.0, 0.0, 0.1),
                     cubic_k1=np.full((2, L, L, L), 0.05, np.float32))


def disk_mask(b: int, L: int, radius: float) -> np.ndarray:
    xs = np.arange(L) - (L - 1) / 2.0
    xg, yg = np.meshgrid(xs, xs, indexing="xy")
    return np.broadcast_to((xg ** 2 + yg ** 2) <= radius ** 2, (b, 1, L, L)).copy()


def xy_ragged_specs(n: int = 96, seed: int = 3, L_min: int = 16, L_max: int = 512):
    """[(crystal, L, disk, T)] of the ragged XY batch."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        crystal = "square" if i < n // 2 else "triangular"
        L = int(round(float(np.exp(rng.uniform(np.log(L_min), np.log(L_max))))))
        T = float(rng.uniform(0.6, 1.2))
        out.append((crystal, L, i % 2 == 1, T))
    return out


def xy_system(crystal: str, L: int, disk: bool) -> sy.System:
    c = cr.make(crystal)
    if disk:
        return sy.System(f"XY {crystal} disk L={L}", 2, c, (L, L), (False, False), {1: 1.0}, h=(0.05, 0.0),
                         mask=disk_mask(c.b, L, 0.45 * L))
    try:
        return sy.System(f"XY {crystal} L={L}", 2, c, (L, L), (True, True), {1: 1.0}, h=(0.05, 0.0))
    except ValueError:
        return sy.System(f"XY {crystal} L={L} (open)", 2, c, (L, L), (False, False), {1: 1.0}, h=(0.05, 0.0))


def xy_angles(system: sy.System, replicas: int, rng: np.random.Generator) -> np.ndarray:
    """(replicas, 2, b, 1, L, L) float32 (cos, sin) of angles uniform in [0, 2 pi); masked sites 0."""
    phi = rng.uniform(0.0, 2.0 * np.pi, size=(replicas,) + system.shape)
    S = np.stack([np.cos(phi), np.sin(phi)], axis=1).astype(np.float32)
    return S * system.site_mask()[None, None].astype(np.float32)
