"""Parity cases shared by the fixture generator and the tests.

Each case builds its System through a factory module `sy` and a crystals module `cr` that expose the
reference's factory API (ising, xy, heisenberg, nanodot, System; make). The fixture generator passes the
reference's own modules, the tests pass this package's, so both sides build the same system from the
same recipe. Sizes are small enough for the reference's CPU path (the Triton interpreter).
"""

from __future__ import annotations

import numpy as np


def _barker(s):
    s.acceptance = "barker"
    return s


def _masked_square(sy, cr):
    rng = np.random.default_rng(0)
    mask = rng.random((1, 1, 8, 8)) > 0.25
    return sy.System("Ising square masked h", 1, cr.make("square"), (8, 8), (True, True), {1: 1.0},
                     h=(0.3,), mask=mask)


def _masked_open_sc(sy, cr):
    mask = np.ones((1, 3, 3, 4), bool)
    mask[0, 1, 1, 1:3] = False
    return sy.System("Ising sc open masked", 1, cr.make("sc"), (4, 3, 3), (False,) * 3, {1: 1.0}, mask=mask)


def heisenberg_bcc_j1j2(sy, cr, L):
    """3D Heisenberg bcc, J1 = 1, J2 = 0.3, cubic K1 = 0.05 on every site, h = 0.1 along z, periodic."""
    c = cr.make("bcc", (1, 2))
    return sy.System("Heisenberg bcc J1-J2", 3, c, (L, L, L), (True,) * 3, {1: 1.0, 2: 0.3},
                     h=(0.0, 0.0, 0.1), cubic_k1=np.full((2, L, L, L), 0.05, np.float32))


def disk_mask(b: int, L: int, radius: float) -> np.ndarray:
    """Circular nanodisk mask of radius `radius` (cells) centred in an L x L box, shape (b, 1, L, L)."""
    xs = np.arange(L) - (L - 1) / 2.0
    xg, yg = np.meshgrid(xs, xs, indexing="xy")
    disk = (xg ** 2 + yg ** 2) <= radius ** 2
    return np.broadcast_to(disk, (b, 1, L, L)).copy()


def xy_disk(sy, cr, crystal, L):
    c = cr.make(crystal)
    return sy.System(f"XY {crystal} disk", 2, c, (L, L), (False, False), {1: 1.0}, h=(0.05, 0.0),
                     mask=disk_mask(c.b, L, 0.45 * L))


def xy_periodic_field(sy, cr, crystal, L):
    c = cr.make(crystal)
    return sy.System(f"XY {crystal} periodic", 2, c, (L, L), (True, True), {1: 1.0}, h=(0.05, 0.0))


# name -> recipe. B replicas, sampler kwargs, base seed, temperature(s), init seed, sweeps.
CASES: dict[str, dict] = {
    # plain int8 / float32 chains (reference tests/test_core.py SMALL, MANY, Barker)
    "ising_square4": dict(build=lambda sy, cr: sy.ising("square", 4), B=2, seed=11, T=1.5, init=2, sweeps=3),
    "xy_square4": dict(build=lambda sy, cr: sy.xy("square", 4), B=2, seed=11, T=1.5, init=2, sweeps=3),
    "heis_bcc2": dict(build=lambda sy, cr: sy.heisenberg("bcc", 2), B=2, seed=11, T=1.5, init=2, sweeps=3),
    "heis_kagome3_afm": dict(build=lambda sy, cr: sy.heisenberg("kagome", 3, J=-1.0), B=2, seed=11, T=1.5,
                             init=2, sweeps=3),
    "nanodot_small": dict(build=lambda sy, cr: sy.nanodot(Rd=2.0, L=2), B=2, seed=11, T=1.5, init=2, sweeps=3),
    "ising_square4_barker": dict(build=lambda sy, cr: _barker(sy.ising("square", 4)), B=2, seed=4, T=1.5,
                                 init=1, sweeps=3),
    "ising_sc5_odd": dict(build=lambda sy, cr: sy.System("Ising sc odd periodic", 1, cr.make("sc"), (5, 5, 5),
                                                          (True,) * 3, {1: 1.0}), B=2, seed=3, T=1.2, init=4,
                          sweeps=3),
    "heis_sc655": dict(build=lambda sy, cr: sy.System("Heisenberg sc 6x5x5 periodic", 3, cr.make("sc"), (6, 5, 5),
                                                       (True,) * 3, {1: 1.0}), B=2, seed=3, T=1.2, init=4, sweeps=3),
    "heis_fcc2": dict(build=lambda sy, cr: sy.heisenberg("fcc", 2), B=2, seed=3, T=1.2, init=4, sweeps=3),
    "xy_sc1055": dict(build=lambda sy, cr: sy.System("XY sc 10x5x5 periodic", 2, cr.make("sc"), (10, 5, 5),
                                                      (True,) * 3, {1: 1.0}), B=2, seed=3, T=1.2, init=4, sweeps=3),
    "heis_triangular6_afm": dict(build=lambda sy, cr: sy.heisenberg("triangular", 6, J=-1.0), B=2, seed=11,
                                 T=1.5, init=2, sweeps=3),
    "xy_sc4": dict(build=lambda sy, cr: sy.xy("sc", 4), B=2, seed=11, T=1.5, init=2, sweeps=3),
    "ising_square8": dict(build=lambda sy, cr: sy.ising("square", 8), B=2, seed=11, T=1.5, init=2, sweeps=3),
    "nanodot_shells": dict(build=lambda sy, cr: sy.nanodot(Rd=2.5, L=3, shells=(1, 2, 4), J_shells={2: 0.3, 4: -0.1}),
                           B=2, seed=3, T=0.5, init=3, sweeps=2),
    "ising_sc_j1j2_field": dict(build=lambda sy, cr: sy.System("Ising sc J1-J2 h", 1, cr.make("sc", (1, 2)), (4, 4, 4),
                                                                (True,) * 3, {1: 1.0, 2: -0.35}, h=(0.2,)),
                                B=4, seed=9, T=[1.5, 2.5, 3.5, 4.5], init=5, sweeps=3),
    "ising_masked_field_barker": dict(build=lambda sy, cr: _barker(_masked_square(sy, cr)), B=3, seed=6,
                                      T=[1.0, 2.0, 3.0], init=2, sweeps=3),
    # packed storage (32 replicas per word, partial last word B = 40) == int8 chain
    "ising_sc_open_packed": dict(build=lambda sy, cr: sy.System("Ising sc open", 1, cr.make("sc"), (4, 3, 3),
                                                                 (False,) * 3, {1: 1.0}),
                                 B=40, seed=5, T=("linspace", 1.5, 4.0, 40), init=9, sweeps=2, packed=True),
    "ising_triangular6_packed": dict(build=lambda sy, cr: sy.ising("triangular", 6), B=40, seed=5,
                                     T=("linspace", 1.5, 4.0, 40), init=9, sweeps=2, packed=True),
    # the workloads at reduced size
    "w1_ising_square32": dict(build=lambda sy, cr: sy.ising("square", 32), B=32, seed=1234,
                              T=("repeat", [1.5, 2.0, 2.269, 3.0], 8), init=0, sweeps=200, packed=False,
                              ref_packed=True, record_every=0),
    "w2_ising_sc8_packed": dict(build=lambda sy, cr: sy.ising("sc", 8), B=64, seed=1,
                                T=("repeat", [4.0, 5.0], 32), init=1, sweeps=3, packed=True),
    "w2_ising_sc8_bitwise": dict(build=lambda sy, cr: sy.ising("sc", 8), B=64, seed=1,
                                 T=("repeat", [4.0, 5.0], 32), init=1, sweeps=3, bitwise=True),
    "w2_ising_sc8_independent": dict(build=lambda sy, cr: sy.ising("sc", 8), B=64, seed=1,
                                     T=("repeat", [4.0, 5.0], 32), init=1, sweeps=3, bitwise=True,
                                     independent=True),
    "w3_heis_bcc4_j1j2": dict(build=lambda sy, cr: heisenberg_bcc_j1j2(sy, cr, 4), B=4, seed=1234,
                              T=("linspace", 0.5, 2.5, 4), init=2, sweeps=10),
    "w4_xy_square16": dict(build=lambda sy, cr: xy_periodic_field(sy, cr, "square", 16), B=2, seed=3, T=0.9,
                           init=3, sweeps=5),
    "w4_xy_triangular12_disk": dict(build=lambda sy, cr: xy_disk(sy, cr, "triangular", 12), B=2, seed=3, T=0.8,
                                    init=3, sweeps=5),
    "w5_ising_sc8": dict(build=lambda sy, cr: sy.ising("sc", 8), B=8, seed=5, T=4.5115, init=3, sweeps=3,
                         packed=False),
}

# bitwise cases of the reference's own exactness test (6 systems x {metropolis, barker}, B = 64, 3 sweeps)
_EXACT = {
    "square8": lambda sy, cr: sy.ising("square", 8),
    "triangular6": lambda sy, cr: sy.ising("triangular", 6),
    "sc4": lambda sy, cr: sy.ising("sc", 4),
    "fcc4": lambda sy, cr: sy.ising("fcc", 4),
    "masked_square": _masked_square,
    "masked_open_sc": _masked_open_sc,
}
_TREF = {"square8": 2.0 / np.log(1 + np.sqrt(2)), "triangular6": 4.0 / np.log(3.0), "sc4": 4.511523, "fcc4": 9.797132}
for _k, _mk in _EXACT.items():
    for _acc in ("metropolis", "barker"):
        for _ind in (False, True):
            def _b(sy, cr, mk=_mk, acc=_acc):
                s = mk(sy, cr)
                s.acceptance = acc
                return s
            tc = _TREF.get(_k, 3.0)
            CASES[f"bw_{_k}_{_acc}{'_ind' if _ind else ''}"] = dict(
                build=_b, B=64, seed=13, T=("list", [2.0 * tc / 3.0] * 32 + [4.0 * tc / 3.0] * 32), init=3,
                sweeps=3, bitwise=True, independent=_ind)


def temperatures(spec, B):
    """Temperature vector of a case as float32 numpy (the reference converts with torch float32)."""
    if isinstance(spec, (int, float)):
        return np.full(B, spec, np.float32)
    if isinstance(spec, list):
        return np.asarray(spec, np.float32)
    kind = spec[0]
    if kind == "linspace":
        import torch
        return torch.linspace(spec[1], spec[2], spec[3]).numpy()
    if kind == "repeat":
        return np.repeat(np.asarray(spec[1], np.float32), spec[2])
    if kind == "list":
        import torch
        return torch.tensor(spec[1]).numpy()
    raise ValueError(spec)


def sampler_kwargs(case: dict) -> dict:
    return {k: case[k] for k in ("packed", "bitwise", "independent", "compact", "max_block") if k in case}


# run-driver cases (tests/test_runs.py; fixtures from make_golden.py runs)
SHAPES = [("sc", (9, 9, 9), "spherical", "r <= 3"), ("sc", (11, 11, 6), "cylindrical", "(rho <= 4) & (abs(z) <= 1.5)"),
          ("bcc", (6, 6, 6), "cartesian", "~((abs(x) < 1) | (abs(y) < 1)) ^ (z > 0)"),
          ("triangular", (12, 10), "cylindrical", "(rho <= 4) & (rho >= 1.5)"),
          ("fcc", (4, 4, 4), "spherical", "(cos(theta) > 0) & (r ** 2 <= 2 * pi)"), ("kagome", (6, 6), "", "")]
THETAS = [("heisenberg", "sc", (7, 7, 3), (False, False, False), "cylindrical", "rho <= 3",
           {"J": {1: 1.0}, "D": 0.88, "K1": 0.177, "Ks": 0.139, "K2": 0.034, "H": 0.483, "H_theta": 30.0,
            "H_phi": 45.0}),
          ("heisenberg", "bcc", (4, 4, 4), (True, True, True), "", "", {"J": {1: 1.0, 2: 0.3}, "K1": 0.05, "H": 0.1}),
          ("xy", "triangular", (6, 6), (True, True), "", "", {"J": {1: 1.0, 2: -0.3}, "H": 0.1, "H_phi": 60.0}),
          ("ising", "square", (37, 5), (True, True), "", "", {"J": {1: 1.0}, "H": 0.2}),
          ("heisenberg", "honeycomb", (6, 6), (True, True), "", "", {"J": {"1": 1.0}, "D": 0.3})]
RUN_CFG = dict(model="ising", crystal="square", box=[6, 6], periodic=[True, True], coords="cylindrical",
               shape="rho <= 2.6", states=[{"name": "a", "J": {"1": 1.0}}, {"name": "b", "J": {"1": 1.0}, "H": 0.2}],
               replicas=5, T_max=3.0, T_min=2.0, T_step=0.5, thermalization=3, measurement=3, measure_every=1,
               units="reduced", seed=1)


def batch_twin_tune(R, resident_limit):
    """Tune sampler R (of one system of a ragged batch) to the path that runs the batch's site update for it: the
    generic resident kernel when the batch keeps the system on-chip, the lattice kernels when the system is on the
    square, triangular or simple cubic table (the batch streams those with the lattice kernels' update), else
    the generic class kernels."""
    if R.sys.nsite * R.sys.n * (1 if R.mode == 0 else 4) <= resident_limit:   # mode 0: int8 storage
        return R.tune(0, 0, resident_limit)
    if R.sys.crystal.name in ("square", "triangular", "sc") and R.tune(1, 0, 0)["specialised"] > 0:
        return R.tune(1, 0, 0)
    return R.tune(0, 0, 0)
