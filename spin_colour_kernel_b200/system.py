"""A system: spin model (n = 1 Ising, 2 XY, 3 Heisenberg), crystal, finite box and couplings.

Spins use the component-planar, basis-planar layout S[B, n, b, L3, L2, L1] with x (L1) fastest; in 2D
L3 = 1. Masked sites hold the zero vector and are never updated, so a masked or open-boundary neighbour
adds nothing to the local field. Validation, the colouring search, the factories and the reference
critical temperatures follow Spin_Colour_Kernel/system.py:19-204; `colour_map` is vectorised.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import crystals as cr
from .colouring import Colouring, search, seam_ok, verify_on_box


@dataclass
class System:
    name: str
    n: int                                   # components per spin (Ising 1, XY 2, Heisenberg 3)
    crystal: cr.Crystal
    box: tuple[int, ...]                     # cells along each lattice axis, x first
    periodic: tuple[bool, ...]
    J: dict[int, float]                      # shell number -> scalar coupling
    extra: dict[int, np.ndarray] = field(default_factory=dict)   # bond position -> added n x n coupling (e.g. DMI)
    h: tuple[float, ...] | None = None       # external field, the same on every site
    cubic_k1: np.ndarray | None = None       # K1 of the cubic anisotropy at every site, (b, L3, L2, L1)
    cubic_k2: float = 0.0                    # K2, multiplying (sx sy sz)^2
    mask: np.ndarray | None = None           # (b, L3, L2, L1) bool, True where a spin lives
    colouring: Colouring | None = None
    T_ref: float | None = None               # known critical temperature of the model, if any
    acceptance: str = "metropolis"           # "metropolis" (u < exp(-beta dE)) or "barker" (u (1 + exp(beta dE)) < 1)

    def __post_init__(self):
        if self.n not in (1, 2, 3):
            raise ValueError("a spin has 1, 2 or 3 components (n)")
        if len(self.box) != self.crystal.D or len(self.periodic) != self.crystal.D:
            raise ValueError("box and periodic need as many entries as the crystal has axes")
        if self.cubic_k1 is not None and self.n != 3:
            raise ValueError("cubic anisotropy is defined for three-component spins only")
        if self.acceptance not in ("metropolis", "barker"):
            raise ValueError("acceptance is 'metropolis' or 'barker'")
        if self.colouring is None:
            self.colouring = search(self.crystal, self.box, self.periodic)
            if self.colouring is None:
                raise ValueError(f"{self.name}: the search found no linear colouring that closes across the seams of box {self.box}")
        if not seam_ok(self.colouring, self.box, self.periodic):
            raise ValueError(f"{self.name}: the colouring does not close across the periodic seams of box {self.box}")
        if not verify_on_box(self.colouring, self.crystal, self.box, self.periodic):
            raise ValueError(f"{self.name}: a bond of the box joins two sites of one colour")

    # ---------------------------------------------------------------- geometry
    @property
    def L1(self) -> int:
        return int(self.box[0])

    @property
    def L2(self) -> int:
        return int(self.box[1])

    @property
    def L3(self) -> int:
        return int(self.box[2]) if self.crystal.D == 3 else 1

    @property
    def b(self) -> int:
        return self.crystal.b

    @property
    def shape(self) -> tuple[int, int, int, int]:
        return (self.b, self.L3, self.L2, self.L1)

    @property
    def nsite(self) -> int:
        return self.b * self.L3 * self.L2 * self.L1

    def site_mask(self) -> np.ndarray:
        return np.ones(self.shape, bool) if self.mask is None else self.mask.astype(bool)

    @property
    def n_active(self) -> int:
        return int(self.site_mask().sum())

    def bond_matrix(self, i: int) -> np.ndarray:
        bd = self.crystal.bonds[i]
        M = self.J.get(bd.shell, 0.0) * np.eye(self.n)
        if i in self.extra:
            M = M + self.extra[i]
        return M

    def colour_map(self) -> np.ndarray:
        """Colour of every site, shape (b, L3, L2, L1), int64."""
        return np.stack([self.colouring.colour_grid(a, tuple(self.box)) for a in range(self.b)])


# -------------------------------------------------------------------- factories
def ising(crystal: str, L: int, J: float = 1.0, shells=(1,), T_ref=None) -> System:
    c = cr.make(crystal, tuple(shells))
    return System(f"Ising {crystal}", 1, c, (L,) * c.D, (True,) * c.D, {s: J for s in shells}, T_ref=T_ref)


def xy(crystal: str, L: int, J: float = 1.0, T_ref=None) -> System:
    c = cr.make(crystal)
    return System(f"XY {crystal}", 2, c, (L,) * c.D, (True,) * c.D, {1: J}, T_ref=T_ref)


def heisenberg(crystal: str, L: int, J: float = 1.0, T_ref=None, label=None) -> System:
    c = cr.make(crystal)
    return System(label or f"Heisenberg {crystal}", 3, c, (L,) * c.D, (True,) * c.D, {1: J}, T_ref=T_ref)


_SC_FIRST_SHELL = ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0))


def nanodot(Rd: float = 18.30, L: int = 5, Jex=1.0, Kan1=0.177, Kan2=0.034, KanS=0.139, Hex=0.483,
            KDM=0.88, gamma_deg=90.0, shells=(1,), J_shells=None) -> System:
    """Simple-cubic Heisenberg disc of radius Rd and L layers inside an open (2N+1)^2 x L box.

    In-plane first-shell bonds carry bulk (Bloch) DMI of strength KDM; sites with fewer than six in-disc
    first neighbours get surface anisotropy KanS instead of Kan1; Kan2 is the (sx sy sz)^2 term and the
    Zeeman field Hex points along (cos g, 0, sin g). Extra shells take couplings J_shells relative to Jex.
    Same Hamiltonian as Spin_Colour_Kernel/system.py:117-171."""
    shells = tuple(sorted(set(shells) | {1}))
    c = cr.make("sc", shells)
    J = {1: Jex, **{int(k): float(v) for k, v in (J_shells or {}).items() if int(k) in shells and int(k) != 1}}
    half = int(Rd) + 1
    N = 2 * half + 1
    xs = np.arange(-half, half + 1)
    xg, yg = np.meshgrid(xs, xs, indexing="xy")
    disk = (xg ** 2 + yg ** 2) <= Rd ** 2                 # indexed [y, x]
    mask = np.broadcast_to(disk, (L, N, N)).copy()[None]  # one sublattice, L layers of the disc
    # in-disc first neighbours per site: y and x wrap (the disc never reaches the edge), z is open
    count = np.zeros(mask.shape[1:], np.int64)
    m3 = mask[0]
    for dz, dy, dx in _SC_FIRST_SHELL:
        shifted = np.roll(m3, shift=(-dy, -dx), axis=(1, 2))
        if dz:
            moved = np.zeros_like(shifted)
            if dz > 0:
                moved[:-1] = shifted[1:]
            else:
                moved[1:] = shifted[:-1]
            shifted = moved
        count += shifted
    surface = (m3 & (count < 6))[None]
    k1 = np.where(surface, KanS, Kan1).astype(np.float32) * mask
    extra = {}
    for i, bd in enumerate(c.bonds):
        E = np.zeros((3, 3))
        d = tuple(bd.delta)
        if d == (1, 0, 0):
            E[1, 2], E[2, 1] = KDM, -KDM
        elif d == (-1, 0, 0):
            E[1, 2], E[2, 1] = -KDM, KDM
        elif d == (0, 1, 0):
            E[0, 2], E[2, 0] = -KDM, KDM
        elif d == (0, -1, 0):
            E[0, 2], E[2, 0] = KDM, -KDM
        if E.any():
            extra[i] = E
    g = np.deg2rad(gamma_deg)
    return System("Heisenberg nanodot", 3, c, (N, N, L), (False, False, False), J, extra,
                  h=(Hex * float(np.cos(g)), 0.0, Hex * float(np.sin(g))), cubic_k1=k1, cubic_k2=Kan2,
                  mask=mask)


# Known critical temperatures in units J = kB = 1 (sources beside each value).
TC = {
    "Ising square": 2.0 / np.log(1 + np.sqrt(2)),
    "Ising triangular": 4.0 / np.log(3.0),
    "Ising sc": 4.511523,      # 1/0.22165463, Ferrenberg, Xu and Landau 2018
    "Ising bcc": 6.355,        # 1/0.157373, Lundow and Campbell 2018
    "Ising fcc": 9.797132,     # 1/0.1020707(2), Yu 2015
    "XY sc": 2.20184,          # 1/0.4541652, Xu et al. 2019
    "Heisenberg sc": 1.4430,   # Chen, Ferrenberg and Landau 1993
    "Heisenberg bcc": 2.0542,  # Chen, Ferrenberg and Landau 1993
}


def matrix(small: bool = True) -> list[System]:
    """The 13 systems of the exactness matrix at a small, seam-compatible size per crystal."""
    return [
        ising("square", 8, T_ref=TC["Ising square"]),
        ising("triangular", 6, T_ref=TC["Ising triangular"]),
        ising("sc", 4, T_ref=TC["Ising sc"]),
        ising("bcc", 4, T_ref=TC["Ising bcc"]),
        ising("fcc", 4, T_ref=TC["Ising fcc"]),
        xy("square", 8, T_ref=0.893),
        xy("sc", 4, T_ref=TC["XY sc"]),
        heisenberg("sc", 4, T_ref=TC["Heisenberg sc"]),
        heisenberg("bcc", 4, T_ref=TC["Heisenberg bcc"]),
        heisenberg("fcc", 4, T_ref=None),
        heisenberg("triangular", 6, J=-1.0, T_ref=0.285, label="Heisenberg triangular AFM"),
        heisenberg("kagome", 6, J=-1.0, T_ref=None, label="Heisenberg kagome AFM"),
        nanodot(Rd=3.0, L=3),
    ]
