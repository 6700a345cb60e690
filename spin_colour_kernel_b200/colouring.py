"""Linear colourings gamma(c, alpha) = K c + o_alpha (mod m) of a crystal's bond graph.

m = (m_1, ..., m_r) is an abelian group in invariant-factor form (m_1 | m_2 | ...), K an r x D integer
matrix and o_alpha one group element per sublattice. A colouring is admissible when no bond joins two
sites of one colour, K delta + o_alpha2 - o_alpha != 0 (mod m) for every bond, and it fits a periodic box
when K[:, k] L_k = 0 (mod m) on every periodic axis k (the seam condition).

The search enumerates groups by increasing order and, inside a group, K columns and offsets in
itertools.product order, returning the first admissible colouring. That order decides WHICH colouring a
system gets and therefore the class order of every sweep, so it follows Spin_Colour_Kernel/colouring.py
:43-100 (`abelian_groups`, `search`) step for step. `verify_on_box` and `colour_map` are vectorised but
decide the same predicate as colouring.py:103-120. The clique number (colouring.py:123-161) certifies
optimality: no colouring can use fewer colours than the largest clique of the bond graph.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np

from .crystals import Crystal


@dataclass(frozen=True)
class Colouring:
    m: tuple[int, ...]                 # group orders, invariant-factor form
    K: tuple[tuple[int, ...], ...]     # r rows of D integers
    o: tuple[tuple[int, ...], ...]     # b rows of r integers

    @property
    def n_colours(self) -> int:
        return int(np.prod(self.m)) if self.m else 1

    def colour(self, c, alpha) -> int:
        """Mixed-radix index of gamma(c, alpha) in [0, n_colours)."""
        idx = 0
        for r, mr in enumerate(self.m):
            g = (sum(self.K[r][k] * int(c[k]) for k in range(len(c))) + self.o[alpha][r]) % mr
            idx = idx * mr + g
        return idx

    def colour_grid(self, alpha: int, box: tuple[int, ...]) -> np.ndarray:
        """Colours of sublattice `alpha` over a whole box, shape (L3, L2, L1) (L3 = 1 in 2D)."""
        D = len(box)
        L = list(box) + [1] * (3 - D)
        z, y, x = np.meshgrid(np.arange(L[2]), np.arange(L[1]), np.arange(L[0]), indexing="ij")
        coords = (x, y, z)
        idx = np.zeros(x.shape, np.int64)
        for r, mr in enumerate(self.m):
            g = np.full(x.shape, self.o[alpha][r], np.int64)
            for k in range(D):
                g = g + int(self.K[r][k]) * coords[k]
            idx = idx * mr + (g % mr)
        return idx

    def describe(self) -> str:
        grp = " x ".join(f"Z{m}" for m in self.m) or "trivial"
        return f"{grp}; K={[list(r) for r in self.K]}; o={[list(x) for x in self.o]}"


def abelian_groups(n: int) -> list[tuple[int, ...]]:
    """Abelian groups of order n as chains m_1 | m_2 | ... | m_r with product n, depth-first by m_1."""
    if n == 1:
        return [()]
    found: list[tuple[int, ...]] = []

    def extend(rest: int, last: int | None, chain: list[int]) -> None:
        if rest == 1:
            found.append(tuple(chain))
            return
        for d in range(2, rest + 1):
            if rest % d == 0 and (last is None or d % last == 0):
                extend(rest // d, d, chain + [d])

    extend(n, None, [])
    return [g for g in found if all(g[i + 1] % g[i] == 0 for i in range(len(g) - 1))]


def _bond_shift(col: Colouring, crystal: Crystal, bd) -> list[int]:
    return [(sum(col.K[r][k] * bd.delta[k] for k in range(crystal.D)) + col.o[bd.alpha2][r] - col.o[bd.alpha][r]) % mr
            for r, mr in enumerate(col.m)]


def admissible(col: Colouring, crystal: Crystal) -> bool:
    """No bond of the table maps to the zero group element."""
    return all(any(v != 0 for v in _bond_shift(col, crystal, bd)) for bd in crystal.bonds)


def seam_ok(col: Colouring, box: tuple[int, ...], periodic: tuple[bool, ...]) -> bool:
    """K[:, k] * L_k = 0 (mod m) on every periodic axis k."""
    for k, (Lk, per) in enumerate(zip(box, periodic)):
        if per and any((col.K[r][k] * Lk) % mr for r, mr in enumerate(col.m)):
            return False
    return True


def search(crystal: Crystal, box: tuple[int, ...] | None = None, periodic: tuple[bool, ...] | None = None,
           max_colours: int = 32) -> Colouring | None:
    """First admissible (and, with a box, seam-compatible) linear colouring by increasing colour count."""
    D, b = crystal.D, crystal.b
    per = periodic or (True,) * D
    for n in range(1, max_colours + 1):
        for m in abelian_groups(n):
            r = len(m)
            elems = list(itertools.product(*[range(mi) for mi in m])) if r else [()]
            zero = tuple([0] * r)
            for cols in itertools.product(elems, repeat=D):
                K = tuple(tuple(cols[k][i] for k in range(D)) for i in range(r))
                for offs in itertools.product(elems, repeat=b - 1):
                    col = Colouring(m, K, (zero,) + tuple(offs))
                    if box is not None and not seam_ok(col, box, per):
                        continue
                    if admissible(col, crystal):
                        return col
    return None


def verify_on_box(col: Colouring, crystal: Crystal, box: tuple[int, ...], periodic: tuple[bool, ...]) -> bool:
    """Colour every site of the box and test every bond explicitly (seam bonds included)."""
    D = crystal.D
    grids = [col.colour_grid(a, box) for a in range(crystal.b)]
    L = list(box) + [1] * (3 - D)
    z, y, x = np.meshgrid(np.arange(L[2]), np.arange(L[1]), np.arange(L[0]), indexing="ij")
    coords = [x, y, z]
    for bd in crystal.bonds:
        if bd.alpha >= crystal.b:
            continue
        inside = np.ones(x.shape, bool)
        nb = []
        for k in range(3):
            q = coords[k] + (bd.delta[k] if k < D else 0)
            if k < D and periodic[k]:
                q = q % L[k]
            else:
                inside &= (q >= 0) & (q < L[k])
                q = np.clip(q, 0, L[k] - 1)
            nb.append(q)
        other = grids[bd.alpha2][nb[2], nb[1], nb[0]]
        if np.any(inside & (grids[bd.alpha] == other)):
            return False
    return True


def clique_number(crystal: Crystal, window: int = 2) -> int:
    """Largest clique of the infinite bond graph (Bron-Kerbosch with pivot-free pruning).

    Any clique can be translated so one of its sites is (0, alpha); its other sites are within one bond
    reach, so a window of that reach around the origin holds every clique."""
    D = crystal.D
    reach = max(max(abs(v) for v in bd.delta) for bd in crystal.bonds)
    w = max(window, reach)
    nodes = [(c, a) for c in itertools.product(range(-w, w + 1), repeat=D) for a in range(crystal.b)]
    where = {nd: i for i, nd in enumerate(nodes)}
    adj: list[set[int]] = [set() for _ in nodes]
    for i, (c, a) in enumerate(nodes):
        for bd in crystal.bonds:
            if bd.alpha != a:
                continue
            j = where.get((tuple(c[k] + bd.delta[k] for k in range(D)), bd.alpha2))
            if j is not None:
                adj[i].add(j)
    best = 1
    for a in range(crystal.b):
        root = where[(tuple([0] * D), a)]

        def expand(R: set, P: set, X: set) -> None:
            nonlocal best
            if not P and not X:
                best = max(best, len(R))
                return
            if len(R) + len(P) <= best:
                return
            for v in list(P):
                expand(R | {v}, P & adj[v], X & adj[v])
                P = P - {v}
                X = X | {v}

        expand({root}, set(adj[root]), set())
    return best
