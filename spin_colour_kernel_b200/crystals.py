"""Bravais lattices with a basis and their directed bond tables.

A site is (c, alpha): an integer cell coordinate c in Z^D and a basis index alpha. A directed bond
(alpha, alpha2, delta, shell) joins (c, alpha) to (c + delta, alpha2). Bonds are found by real-space
distance: shell s is the s-th smallest non-zero distance between any two basis sites within `reach`
cells.

The table order is part of the contract, because it is the accumulation order of the float32 local
field in every kernel: shell ascending, then alpha, then alpha2, then delta in lexicographic order
with the last lattice axis varying fastest. This follows Spin_Colour_Kernel/crystals.py:48-101
(`shell_distances`, `build_bonds`, `make`).
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

#: the crystals of the reference's system matrix: (lattice vectors as rows, basis in cell coordinates)
_SQRT3 = float(np.sqrt(3.0))
_TRI = ((1.0, 0.0), (0.5, _SQRT3 / 2))
LATTICES: dict[str, tuple[tuple, tuple]] = {
    "square": (((1.0, 0.0), (0.0, 1.0)), ((0.0, 0.0),)),
    "triangular": (_TRI, ((0.0, 0.0),)),
    "honeycomb": (_TRI, ((0.0, 0.0), (1 / 3, 1 / 3))),
    "kagome": (_TRI, ((0.0, 0.0), (0.5, 0.0), (0.0, 0.5))),
    "sc": (((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)), ((0.0, 0.0, 0.0),)),
    "bcc": (((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)), ((0.0, 0.0, 0.0), (0.5, 0.5, 0.5))),
    "fcc": (((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)),
            ((0.0, 0.0, 0.0), (0.5, 0.5, 0.0), (0.5, 0.0, 0.5), (0.0, 0.5, 0.5))),
}


@dataclass(frozen=True)
class Bond:
    """Directed bond (c, alpha) -> (c + delta, alpha2) on neighbour shell `shell` (1-based)."""

    alpha: int
    alpha2: int
    delta: tuple[int, ...]
    shell: int


@dataclass
class Crystal:
    name: str
    vectors: np.ndarray          # (D, D): row k is lattice vector a_k (Cartesian)
    basis: np.ndarray            # (b, D): basis offsets in cell coordinates
    shells: tuple[int, ...] = (1,)
    bonds: list[Bond] = field(default_factory=list)

    @property
    def D(self) -> int:
        return int(self.vectors.shape[0])

    @property
    def b(self) -> int:
        return int(self.basis.shape[0])

    def position(self, c, alpha) -> np.ndarray:
        return (np.asarray(c, dtype=float) + self.basis[alpha]) @ self.vectors


def _separation(vectors: np.ndarray, basis: np.ndarray, a: int, a2: int, delta) -> float:
    """Euclidean length of the bond (0, a) -> (delta, a2)."""
    r = (np.asarray(delta, float) + basis[a2] - basis[a]) @ vectors
    return float(np.linalg.norm(r))


def _deltas(D: int, reach: int):
    """Every cell offset with components in [-reach, reach], lexicographic (last axis fastest)."""
    return itertools.product(range(-reach, reach + 1), repeat=D)


def shell_distances(vectors: np.ndarray, basis: np.ndarray, nshell: int, reach: int = 3) -> list[float]:
    """The `nshell` smallest distinct non-zero site separations (rounded to 1e-9)."""
    found: set[float] = set()
    nb = basis.shape[0]
    for a in range(nb):
        for a2 in range(nb):
            for delta in _deltas(vectors.shape[0], reach):
                d = _separation(vectors, basis, a, a2, delta)
                if d > 1e-9:
                    found.add(round(d, 9))
    return sorted(found)[:nshell]


def build_bonds(vectors: np.ndarray, basis: np.ndarray, shells: tuple[int, ...], reach: int = 3) -> list[Bond]:
    """Directed bonds of the requested shells in table order (shell, alpha, alpha2, delta)."""
    radii = shell_distances(vectors, basis, max(shells), reach)
    nb, D = basis.shape[0], vectors.shape[0]
    table: list[Bond] = []
    for s in sorted(shells):
        want = radii[s - 1]
        for a in range(nb):
            for a2 in range(nb):
                for delta in _deltas(D, reach):
                    if abs(_separation(vectors, basis, a, a2, delta) - want) < 1e-7:
                        table.append(Bond(a, a2, tuple(int(v) for v in delta), s))
    return table


def make(name: str, shells: tuple[int, ...] = (1,)) -> Crystal:
    """Crystal `name` with the bonds of `shells`; bcc and fcc use the conventional cubic cell."""
    if name not in LATTICES:
        raise KeyError(f"unknown crystal {name!r}; known: {sorted(LATTICES)}")
    vec, basis = (np.asarray(x, float) for x in LATTICES[name])
    shells = tuple(shells)
    reach = 3 if max(shells) <= 2 else 4
    return Crystal(name, vec, basis, shells, build_bonds(vec, basis, shells, reach))


def coordination(crystal: Crystal) -> dict[int, int]:
    """Number of bonds leaving each sublattice."""
    out = {a: 0 for a in range(crystal.b)}
    for bd in crystal.bonds:
        out[bd.alpha] += 1
    return out
