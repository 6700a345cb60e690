"""Interleaved ('quad') storage of vector models: four replicas per float4, rows split by colour residue.

The interleaved class kernels run the same packed-pair arithmetic as the lattice kernels of the reference layout,
so their chains must be identical to those kernels' spin for spin (bit-exact), and within the vector-model
tolerance of the reference's recorded chains. Conversions must round-trip exactly; FP64 observables read from
the quads must equal those of the reference layout.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

import cases as C
from oracle import observables as obs
from spin_colour_kernel_b200 import _lib as L
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import system as sy

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
VEC_TOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200 import build
    build.build()


def _quad(s, B, seed=1, **kw):
    from spin_colour_kernel_b200.sampler import Sampler
    return Sampler(s, B, device="cuda", seed=seed, layout="quad", **kw)


def _supported(s):
    """Whether the library accepts an interleaved plan for this system (a host-only call)."""
    import ctypes
    from spin_colour_kernel_b200 import plan as P
    d = P.describe(s)
    h = ctypes.c_void_p()
    rc = L.lib().sck_plan_create(ctypes.byref(d), 4, L.MODE_QUAD, ctypes.byref(h))
    if rc == L.OK:
        L.lib().sck_plan_destroy(h)
    return rc == L.OK


VEC_FIXTURES = [k for k in C.CASES if (GOLD / f"{k}.npz").exists() and not C.CASES[k].get("bitwise")
                and C.CASES[k]["build"](sy, cr).n > 1]


@pytest.mark.parametrize("name", VEC_FIXTURES)
def test_quad_chain_matches_reference_fixture(name):
    case = C.CASES[name]
    s = case["build"](sy, cr)
    if not _supported(s):
        with pytest.raises(ValueError):
            _quad(s, case["B"], seed=case["seed"])
        return
    g = dict(np.load(GOLD / f"{name}.npz"))
    A = _quad(s, case["B"], seed=case["seed"])
    A.set_temperature(torch.from_numpy(g["T"]))
    S = A.init_spins(seed=case["init"])
    assert np.array_equal(A.unpack(S).cpu().numpy(), g["S0"]), "initial spins differ"
    snaps = {int(k): i for i, k in enumerate(g["snap_ids"])}
    for k in range(1, case["sweeps"] + 1):
        A.sweep(S)
        if k in snaps:
            got = A.unpack(S).cpu().numpy().astype(np.float64)
            d = np.abs(got - g["snaps"][snaps[k]].astype(np.float64))
            frac = float((d > VEC_TOL).any(axis=1).mean())
            assert frac <= 0.02, f"{name}: {frac:.4f} of spins beyond {VEC_TOL}"
    assert int(A.state[1]) == case["sweeps"]


def test_quad_fixture_coverage():
    """The interleaved path serves the periodic lattice-table fixtures the workloads need."""
    served = [k for k in VEC_FIXTURES if _supported(C.CASES[k]["build"](sy, cr))]
    for need in ("w3_heis_bcc4_j1j2", "w4_xy_square16", "heis_bcc2", "heis_fcc2", "xy_square4"):
        assert need in served, need


SYSTEMS = [
    ("bcc J1-J2 K1 h 8^3", lambda: C.heisenberg_bcc_j1j2(sy, cr, 8), 10),
    ("bcc J1-J2 K1 h 6^3 odd replicas", lambda: C.heisenberg_bcc_j1j2(sy, cr, 6), 7),
    ("Heisenberg sc 8x6x4 h", lambda: sy.System("Heisenberg sc", 3, cr.make("sc"), (8, 6, 4), (True,) * 3,
                                               {1: -1.0}, h=(0.1, 0.0, 0.2)), 8),
    ("Heisenberg fcc 4^3", lambda: sy.heisenberg("fcc", 4), 5),
    ("Heisenberg bcc J1 4^3", lambda: sy.heisenberg("bcc", 4), 6),
    ("XY square 16 h", lambda: C.xy_periodic_field(sy, cr, "square", 16), 9),
    ("XY triangular 8", lambda: sy.xy("triangular", 8), 4),
    ("XY sc 64x4x4 (templated row)", lambda: sy.System("XY sc", 2, cr.make("sc"), (64, 4, 4), (True,) * 3,
                                                       {1: 1.0}), 4),
    ("Heisenberg bcc J1-J2 32x4x4 Barker", lambda: _barker(sy.System(
        "Heisenberg bcc", 3, cr.make("bcc", (1, 2)), (32, 4, 4), (True,) * 3, {1: 1.0, 2: 0.3})), 8),
]


def _barker(s):
    s.acceptance = "barker"
    return s


@pytest.mark.parametrize("label, make, B", SYSTEMS, ids=[x[0] for x in SYSTEMS])
def test_quad_sweeps_equal_lattice_kernels_bit_for_bit(label, make, B):
    from spin_colour_kernel_b200.sampler import Sampler
    s = make()
    R = Sampler(s, B, device="cuda", seed=77)
    R.tune(1, 0, 0)                    # lattice kernels, class by class (no resident or tile path)
    Q = _quad(s, B, seed=77)
    T = torch.linspace(0.4, 3.0, B)
    R.set_temperature(T)
    Q.set_temperature(T)
    X = R.init_spins(seed=5)
    S = Q.pack(X)
    assert torch.equal(Q.unpack(S), X)
    for k in range(4):
        R.sweep(X, 1 + k)
        Q.sweep(S, 1 + k)
        assert torch.equal(Q.unpack(S), X), f"{label}: sweep block {k}"
    assert int(Q.state[1]) == int(R.state[1]) == 10


def test_quad_pack_round_trip_and_padding():
    s = C.heisenberg_bcc_j1j2(sy, cr, 4)
    Q = _quad(s, 6)
    x = torch.randn((6, 3) + s.shape, device="cuda")
    S = Q.pack(x)
    assert tuple(S.shape) == (2, 2, 4, 4, 3, 4, 4)
    assert torch.equal(Q.unpack(S), x)
    # lanes 2, 3 of the last quad are padding, zero after a pack
    assert torch.count_nonzero(S[1, ..., 2:]) == 0
    # element order: component k of site (a, z, y, x) at [q, a, z, y, k, (x % 2) * 2 + x // 2, j]
    xn, Sn = x.cpu().numpy(), S.cpu().numpy()
    for (rep, k, a, z, y, xx) in [(0, 0, 0, 0, 0, 0), (5, 2, 1, 3, 2, 3), (2, 1, 0, 1, 3, 2), (3, 0, 1, 2, 0, 1)]:
        assert Sn[rep // 4, a, z, y, k, (xx % 2) * 2 + xx // 2, rep % 4] == xn[rep, k, a, z, y, xx]


def test_quad_observables_equal_reference_layout_and_oracle():
    for s, B in ((C.heisenberg_bcc_j1j2(sy, cr, 6), 7), (C.xy_periodic_field(sy, cr, "square", 16), 5),
                 (sy.heisenberg("fcc", 4), 4)):
        Q = _quad(s, B, seed=3)
        Q.set_temperature(torch.linspace(0.5, 2.0, B))
        S = Q.init_spins(seed=3)
        Q.sweep(S, 2)
        E, M = Q.observables(S)
        x = Q.unpack(S)
        E2, M2 = Q._flat().observables(x)
        np.testing.assert_allclose(E.cpu().numpy(), E2.cpu().numpy(), rtol=1e-12, atol=1e-9, err_msg=s.name)
        np.testing.assert_allclose(M.cpu().numpy(), M2.cpu().numpy(), rtol=1e-12, atol=1e-9, err_msg=s.name)
        xn = x.cpu().numpy()
        np.testing.assert_allclose(E.cpu().numpy(), obs.energy(s, xn), rtol=1e-12, atol=1e-9, err_msg=s.name)
        np.testing.assert_allclose(M.cpu().numpy(), obs.magnetization(xn), rtol=1e-12, atol=1e-9)


def test_quad_graph_replay_equals_sweeps():
    s = C.heisenberg_bcc_j1j2(sy, cr, 8)
    A, B = _quad(s, 8, seed=9), _quad(s, 8, seed=9)
    for X in (A, B):
        X.set_temperature(torch.linspace(0.5, 2.5, 8))
    S1, S2 = A.init_spins(seed=1), B.init_spins(seed=1)
    rep = A.graph(S1, 3)       # one warm-up sweep, then a graph of 3
    rep()
    B.sweep(S2, 4)
    assert torch.equal(S1, S2)


def test_quad_reference_sweep_and_sync_control_match_reference_layout():
    from spin_colour_kernel_b200.sampler import Sampler
    s = sy.heisenberg("bcc", 2)
    Q = _quad(s, 3, seed=11)
    R = Sampler(s, 3, device="cuda", seed=11)
    for X in (Q, R):
        X.set_temperature(1.5)
    x = R.init_spins(seed=2)
    S = Q.pack(x)
    R.reference_sweep(x, 2)
    Q.reference_sweep(S, 2)
    assert torch.equal(Q.unpack(S), x)
    assert int(Q.state[1]) == 2


def test_quad_refuses_unsupported_systems():
    with pytest.raises(ValueError):
        _quad(sy.ising("square", 8), 4)                       # Ising
    with pytest.raises(ValueError):
        _quad(C.xy_disk(sy, cr, "square", 12), 4)             # mask, open boundary
    with pytest.raises(ValueError):
        _quad(sy.heisenberg("triangular", 6), 4)              # colouring of x-period 3
    with pytest.raises(ValueError):
        _quad(sy.heisenberg("kagome", 4), 4)                  # no compile-time lattice table


@pytest.mark.parametrize("make, B", [(lambda: C.heisenberg_bcc_j1j2(sy, cr, 8), 10),
                                     (lambda: C.xy_periodic_field(sy, cr, "square", 16), 6),
                                     (lambda: sy.heisenberg("fcc", 4), 4),
                                     (lambda: sy.heisenberg("bcc", 4), 8)])
def test_measure_sweep_equals_sweep_then_observables(make, B):
    """The fused measure step leaves the same chain as plain sweeps, and its observables equal the FP64 pass on
    the state it leaves: magnetizations to FP64 rounding, energies to the float32 rounding of the site shares."""
    s = make()
    A, R = _quad(s, B, seed=13), _quad(s, B, seed=13)
    for X in (A, R):
        X.set_temperature(torch.linspace(0.6, 2.6, B))
    S1, S2 = A.init_spins(seed=4), R.init_spins(seed=4)
    for n in (1, 3):
        E, M = A.sweep_measure(S1, n)
        R.sweep(S2, n)
        assert torch.equal(S1, S2)
        E2, M2 = R.observables(S2)
        np.testing.assert_allclose(M.cpu().numpy(), M2.cpu().numpy(), rtol=1e-11, atol=1e-9, err_msg=s.name)
        np.testing.assert_allclose(E.cpu().numpy(), E2.cpu().numpy(), rtol=2e-6, atol=1e-5 * s.n_active,
                                   err_msg=s.name)
    assert int(A.state[1]) == int(R.state[1]) == 4


def test_measure_sweep_graph_capture():
    s = C.heisenberg_bcc_j1j2(sy, cr, 8)
    A = _quad(s, 8, seed=2)
    A.set_temperature(torch.linspace(0.5, 2.5, 8))
    S = A.init_spins(seed=1)
    E = torch.empty(8, dtype=torch.float64, device="cuda")
    M = torch.empty((8, 2, 3), dtype=torch.float64, device="cuda")
    A.sweep_measure(S, 1, E, M)                          # first call: sizes the workspace
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        A.sweep_measure(S, 2, E, M)
    g.replay()
    E2, M2 = A.observables(S)
    np.testing.assert_allclose(E.cpu().numpy(), E2.cpu().numpy(), rtol=2e-6)
    np.testing.assert_allclose(M.cpu().numpy(), M2.cpu().numpy(), rtol=1e-11, atol=1e-9)
    assert int(A.state[1]) == 3


def test_measure_step_of_reference_layout_is_sweep_then_observables():
    from spin_colour_kernel_b200.sampler import Sampler
    s = C.xy_periodic_field(sy, cr, "square", 16)
    A, R = Sampler(s, 5, device="cuda", seed=3), Sampler(s, 5, device="cuda", seed=3)
    for X in (A, R):
        X.set_temperature(0.8)
    S1, S2 = A.init_spins(seed=2), R.init_spins(seed=2)
    E, M = A.sweep_measure(S1, 2)
    R.sweep(S2, 2)
    E2, M2 = R.observables(S2)
    assert torch.equal(S1, S2) and torch.equal(E, E2) and torch.equal(M, M2)


PIPE_CASES = [
    ("bcc J1-J2 8^3, 40 replicas, groups of 8, skew 1", lambda: C.heisenberg_bcc_j1j2(sy, cr, 8), 40, 8, 1),
    ("bcc J1-J2 8^3, 38 replicas, groups of 12, skew 2", lambda: C.heisenberg_bcc_j1j2(sy, cr, 8), 38, 12, 2),
    ("bcc J1-J2 8^3, 24 replicas, groups of 4, skew 4", lambda: C.heisenberg_bcc_j1j2(sy, cr, 8), 24, 4, 4),
    ("bcc J1-J2 64x8x8, 16 replicas, groups of 4, skew 2", lambda: sy.System(
        "Heisenberg bcc", 3, cr.make("bcc", (1, 2)), (64, 8, 8), (True,) * 3, {1: 1.0, 2: 0.3}), 16, 4, 2),
    ("XY square 32 h, 20 replicas, groups of 4, skew 1", lambda: C.xy_periodic_field(sy, cr, "square", 32), 20, 4,
     1),
    ("Heisenberg fcc 4^3, 16 replicas, groups of 4, skew 2", lambda: sy.heisenberg("fcc", 4), 16, 4, 2),
]


@pytest.mark.parametrize("label, make, B, group, skew", PIPE_CASES, ids=[x[0] for x in PIPE_CASES])
def test_pipeline_equals_class_by_class(label, make, B, group, skew):
    """The class-skewed L2 pipeline only reorders independent work: spins identical to class-by-class launches,
    over several calls of several sweeps (partial last groups, padding lanes, every skew that divides the class
    count)."""
    s = make()
    A, R = _quad(s, B, seed=21), _quad(s, B, seed=21)
    path = A.pipeline(group, skew)
    assert path["group"] == group
    for X in (A, R):
        X.set_temperature(torch.linspace(0.5, 3.0, B))
    S1, S2 = A.init_spins(seed=8), R.init_spins(seed=8)
    for n in (1, 3, 2):
        A.sweep(S1, n)
        R.sweep(S2, n)
        assert torch.equal(S1, S2), label
    A.check_waits()
    assert int(A.state[1]) == 6


@pytest.mark.parametrize("chunks", [1, 3, 64])
def test_pipeline_ticket_size_does_not_change_the_chain(chunks):
    """Tickets of 1, 3 (a partial last ticket per quad and class) and 64 site blocks (one ticket per quad and
    class): the same spins as class-by-class launches, and the same measure-step observables."""
    s = sy.System("Heisenberg bcc", 3, cr.make("bcc", (1, 2)), (32, 16, 16), (True,) * 3, {1: 1.0, 2: 0.3},
                  h=(0.0, 0.0, 0.1))
    B = 20
    A, R = _quad(s, B, seed=5), _quad(s, B, seed=5)
    A.pipeline(4, 2, chunks)
    for X in (A, R):
        X.set_temperature(torch.linspace(0.5, 3.0, B))
    S1, S2 = A.init_spins(seed=3), R.init_spins(seed=3)
    A.sweep(S1, 3)
    R.sweep(S2, 3)
    assert torch.equal(S1, S2)
    E1, M1 = A.sweep_measure(S1, 2)
    E2, M2 = R.sweep_measure(S2, 2)
    assert torch.equal(S1, S2)
    np.testing.assert_allclose(E1.cpu().numpy(), E2.cpu().numpy(), rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(M1.cpu().numpy(), M2.cpu().numpy(), rtol=1e-12, atol=1e-9)
    A.check_waits()
    with pytest.raises(ValueError):
        A.pipeline(4, 2, 0)


def test_pipeline_refuses_bad_groups_and_skews():
    s = C.heisenberg_bcc_j1j2(sy, cr, 8)          # 4 classes
    A = _quad(s, 16, seed=1)
    for group, skew in ((6, 2), (8, 3), (16, 1), (-4, 2)):   # not whole quads, skew not dividing 4, too few groups
        with pytest.raises(ValueError):
            A.pipeline(group, skew)
    from spin_colour_kernel_b200.sampler import Sampler
    with pytest.raises(ValueError):
        Sampler(s, 16, device="cuda").pipeline(8, 2)           # the reference layout takes an L2 budget instead


def test_pipeline_wait_that_gives_up_reports_timeout():
    """A wait limit shortened to one poll makes blocks give up instead of waiting for the class they follow: the
    kernel returns normally (no trap, nothing hangs), the sweep's sites are partly left unchanged, and the plan
    reports SCK_ERR_TIMEOUT: sck_sweep refuses until the status is read, the status read clears it, and with the
    default limit restored the pipeline again equals class-by-class launches."""
    from spin_colour_kernel_b200 import _lib as L
    s = sy.System("Heisenberg bcc", 3, cr.make("bcc", (1, 2)), (32, 32, 16), (True,) * 3, {1: 1.0, 2: 0.3})
    A = _quad(s, 32, seed=3)
    A.pipeline(32, 4)                              # one group, classes strictly in sequence: every class waits
    A.set_temperature(1.0)
    S = A.init_spins(seed=1)
    A.set_wait_limit(1)
    A.sweep(S, 2)
    torch.cuda.synchronize()
    with pytest.raises(L.SckError) as e:
        A.sweep(S, 1)                              # refused: an earlier wait of this plan gave up
    assert e.value.code == L.ERR_TIMEOUT
    with pytest.raises(L.SckError) as e:
        A.check_waits()
    assert e.value.code == L.ERR_TIMEOUT
    A.check_waits()                                # cleared
    A.set_wait_limit(1 << 20)
    R = _quad(s, 32, seed=3)
    R.set_temperature(1.0)
    X = S.clone()
    A.state.copy_(R.state)
    A.sweep(S, 2)
    R.sweep(X, 2)
    A.check_waits()
    assert torch.equal(S, X)


@pytest.mark.parametrize("B, group, skew", [(24, 4, 2), (22, 4, 1), (16, 4, 4)])
def test_pipeline_measure_step_equals_sweeps_then_observables(B, group, skew):
    """A measure step through the pipeline (its last sweep accumulating the FP64 sums) leaves the chain of
    class-by-class sweeps and returns the observables of the state it leaves."""
    s = C.heisenberg_bcc_j1j2(sy, cr, 8)
    A, R = _quad(s, B, seed=17), _quad(s, B, seed=17)
    A.pipeline(group, skew)
    for X in (A, R):
        X.set_temperature(torch.linspace(0.5, 2.5, B))
    S1, S2 = A.init_spins(seed=2), R.init_spins(seed=2)
    for n in (1, 4):
        E, M = A.sweep_measure(S1, n)
        R.sweep(S2, n)
        assert torch.equal(S1, S2)
        E2, M2 = R.observables(S2)
        np.testing.assert_allclose(M.cpu().numpy(), M2.cpu().numpy(), rtol=1e-11, atol=1e-9)
        np.testing.assert_allclose(E.cpu().numpy(), E2.cpu().numpy(), rtol=2e-6, atol=1e-5 * s.n_active)
    A.check_waits()


def test_autotuned_schedule_is_bit_identical_and_cached(tmp_path, monkeypatch):
    """The autotuner times class-by-class launches against every pipeline group and class skew, applies the
    fastest, caches it per system, and the tuned path leaves the chain of the default path."""
    from spin_colour_kernel_b200 import autotune as at
    monkeypatch.setenv("SCK_TUNE_CACHE", str(tmp_path / "tune.json"))
    s = C.heisenberg_bcc_j1j2(sy, cr, 16)
    A, R = _quad(s, 64, seed=31), _quad(s, 64, seed=31)
    for X in (A, R):
        X.set_temperature(torch.linspace(0.5, 2.5, 64))
    S1, S2 = A.init_spins(seed=1), R.init_spins(seed=1)
    c = at.autotune(A, S1, sweeps=2)
    assert not c["cached"] and len(c["tried"]) == len(at.quad_candidates(A)) > 4
    assert int(A.state[1]) == 0                        # the counter is restored
    A.sweep(S1, 3)
    R.sweep(S2, 3)
    assert torch.equal(S1, S2)
    B = _quad(s, 64, seed=31)
    c2 = at.autotune(B, B.init_spins(seed=1))
    assert c2["cached"] and (c2["group"], c2["skew"], c2["chunks"]) == (c["group"], c["skew"], c["chunks"])
    assert B.path()["group"] == c["group"]


def test_autotuned_batch_is_bit_identical_and_cached(tmp_path, monkeypatch):
    """The batch autotuner times the persistent batch kernel at several resident limits (which systems run
    on-chip), restores every counter, returns the fastest batch, caches the choice, and the tuned batch continues
    the chains of the systems swept on their own."""
    from spin_colour_kernel_b200 import autotune as at
    from spin_colour_kernel_b200 import workloads as W
    from spin_colour_kernel_b200.sampler import Sampler
    monkeypatch.setenv("SCK_TUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(9)
    specs = [("square", 16, False, 0.7), ("triangular", 45, True, 1.0), ("square", 96, False, 0.9)]
    samplers, spins, refs, ref_spins = [], [], [], []
    for i, (crystal, L, disk, T) in enumerate(specs):
        s = W.xy_system(crystal, L, disk)
        A, R = Sampler(s, 4, device="cuda", seed=70 + i), Sampler(s, 4, device="cuda", seed=70 + i)
        for X in (A, R):
            X.set_temperature(T)
        S = torch.from_numpy(W.xy_angles(s, 4, rng)).cuda()
        samplers += [A]
        spins += [S]
        refs += [R]
        ref_spins += [S.clone()]
    batch, c = at.autotune_batch(samplers, spins, sweeps=2)
    assert not c["cached"] and len(c["tried"]) >= 2
    for R in refs:
        C.batch_twin_tune(R, c["resident_limit"])
    assert all(int(A.state[1]) == 0 for A in samplers)
    batch.sweep(3)
    for R, S in zip(refs, ref_spins):
        R.sweep(S, 3)
    for S, S2 in zip(spins, ref_spins):
        assert torch.equal(S, S2)
    _, c2 = at.autotune_batch(samplers, spins)
    assert c2["cached"] and c2["resident_limit"] == c["resident_limit"]
