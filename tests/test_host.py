"""Host-side logic, without a GPU: the C-ABI library, the system lowering, the host-built acceptance tables
and the Sampler's argument checks."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import cases as C
from oracle import philox
from oracle import sweep as osw
from spin_colour_kernel_b200 import _lib as L
from spin_colour_kernel_b200 import colouring as co
from spin_colour_kernel_b200 import crystals as cr
from spin_colour_kernel_b200 import plan as P
from spin_colour_kernel_b200 import system as sy

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"


@pytest.fixture(scope="module", autouse=True)
def _built():
    from spin_colour_kernel_b200 import build
    build.build()


def test_library_exports_every_declared_symbol():
    decl = set()
    for h in (ROOT / "include").glob("*.h"):
        decl |= set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(sck_\w+)\s*\(", h.read_text(), re.M))
    assert decl, "no declarations found"
    lib = L.lib()
    missing = [s for s in sorted(decl) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(L.EXPORTS) <= decl


def test_struct_layout_matches_binding():
    L.lib()          # raises on a size mismatch


def _plan(s, batch, mode):
    d = P.describe(s)
    h = ctypes.c_void_p()
    rc = L.lib().sck_plan_create(ctypes.byref(d), batch, mode, ctypes.byref(h))
    if rc == 0:
        L.lib().sck_plan_destroy(h)
    return rc, L.lib().sck_last_error().decode()


def test_plan_refusals_mirror_the_reference():
    assert _plan(sy.ising("sc", 4), 64, L.MODE_BITWISE)[0] == 0
    assert _plan(sy.heisenberg("sc", 4), 32, L.MODE_BITWISE)[0] == L.ERR_UNSUPPORTED
    assert _plan(sy.heisenberg("sc", 4), 32, L.MODE_PACKED)[0] == L.ERR_UNSUPPORTED
    rc, msg = _plan(sy.ising("sc", 128), 1024, L.MODE_BITWISE)
    assert rc == L.ERR_COUNTER and "Philox" in msg
    assert _plan(sy.ising("sc", 128), 512, L.MODE_BITWISE)[0] == 0
    s = sy.System("J1-J2", 1, cr.make("sc", (1, 2)), (4, 4, 4), (True,) * 3, {1: 1.0, 2: 0.5})
    assert _plan(s, 32, L.MODE_BITWISE)[0] == L.ERR_UNSUPPORTED
    assert _plan(s, 32, L.MODE_INT8)[0] == 0
    d = P.describe(sy.ising("square", 4))
    d.abi_version = 99
    h = ctypes.c_void_p()
    assert L.lib().sck_plan_create(ctypes.byref(d), 4, L.MODE_INT8, ctypes.byref(h)) == L.ERR_INVALID


def test_interleaved_plans_accept_the_periodic_lattice_table_systems_only():
    bcc = C.heisenberg_bcc_j1j2(sy, cr, 64)
    assert _plan(bcc, 1536, L.MODE_QUAD)[0] == 0
    shape = ctypes.c_int32(), ctypes.c_int32()
    d = P.describe(bcc)
    h = ctypes.c_void_p()
    assert L.lib().sck_plan_create(ctypes.byref(d), 7, L.MODE_QUAD, ctypes.byref(h)) == 0
    L.lib().sck_plan_shape(h, ctypes.byref(shape[0]), ctypes.byref(shape[1]))
    L.lib().sck_plan_destroy(h)
    assert (shape[0].value, shape[1].value) == (8, 2)           # 7 replicas computed as 2 quads
    for s in (sy.xy("square", 16), sy.heisenberg("fcc", 4), sy.heisenberg("bcc", 4), sy.xy("triangular", 8)):
        assert _plan(s, 4, L.MODE_QUAD)[0] == 0, s.name
    for s, word in ((sy.ising("square", 8), "vector"), (C.xy_disk(sy, cr, "square", 12), "mask"),
                    (sy.heisenberg("triangular", 6), "x-period"), (sy.heisenberg("kagome", 4), "table"),
                    (sy.System("XY sc open", 2, cr.make("sc"), (4, 4, 4), (False,) * 3, {1: 1.0}), "periodic")):
        rc, msg = _plan(s, 4, L.MODE_QUAD)
        assert rc == L.ERR_UNSUPPORTED and word in msg, (s.name, msg)
    # the Philox envelope counts the padding lanes: 4 * ceil(B / 4) replicas
    assert _plan(bcc, 4096, L.MODE_QUAD)[0] == L.ERR_COUNTER


def test_describe_groups_bonds_by_coupling_in_first_appearance_order():
    # shells 1 and 3 share J: one group of 6 + 8 bonds, then shell 2 (12 bonds); J = 0 shell 4 is left out
    s = sy.System("sc shells", 1, cr.make("sc", (1, 2, 3, 4)), (9, 9, 9), (True,) * 3,
                  {1: 1.0, 2: 0.25, 3: 1.0, 4: 0.0})
    d = P.describe(s)
    sub = d.sub[0]
    assert sub.n_groups == 2 and list(sub.group_end[:2]) == [14, 26] and sub.n_bonds == 26
    assert list(sub.group_J[:2]) == [1.0, 0.25]
    order = [b for b in s.crystal.bonds if b.shell in (1, 3)] + [b for b in s.crystal.bonds if b.shell == 2]
    got = [(sub.bonds[i].alpha2, tuple(sub.bonds[i].d)) for i in range(26)]
    assert got == [(b.alpha2, tuple(b.delta)) for b in order]


def _emulate_ising_class(s, S, table, keys, base_seed, sweep, colour, alpha):
    """The kernels' Ising update in NumPy: integer key -> table -> compare with the uniform."""
    b, L3, L2, L1 = s.shape
    nsite = b * L3 * L2 * L1
    B = S.shape[0]
    mask = s.site_mask()
    z, y, x = np.nonzero((s.colour_map()[alpha] == colour) & mask[alpha])
    own = alpha * L3 * L2 * L1 + z * L2 * L1 + y * L1 + x
    d = P.describe(s).sub[alpha]
    si = np.sign(S[:, 0, alpha, z, y, x]).astype(np.int64)
    k = (si > 0).astype(np.int64)
    stride = 2
    bi = 0
    for g in range(d.n_groups):
        G = np.zeros_like(si)
        for _ in range(bi, d.group_end[g]):
            bd = d.bonds[bi]
            zq, yq, xq, ok = osw.neighbour(s, type("B", (), {"delta": tuple(bd.d)[: s.crystal.D]}), z, y, x)
            G += np.where(ok[None, :], np.sign(S[:, 0, bd.alpha2, zq, yq, xq]).astype(np.int64), 0)
            bi += 1
        if d.group_apply[g]:
            zg = d.group_end[g] - (d.group_end[g - 1] if g else 0)
            k += (G + zg) * stride
            stride *= 2 * zg + 1
    e = table[np.arange(B)[:, None], alpha, k]
    key = int(np.int64(philox.sweep_seed(base_seed, sweep)).astype(np.int32))
    ctr = philox.int32_counter(np.arange(B, dtype=np.int64)[:, None] * nsite + own[None, :])
    u0 = philox.uniform4(key, ctr.reshape(-1))[0].reshape(B, -1)
    if s.acceptance == "barker":
        acc = u0 * (np.float32(1.0) + e) < np.float32(1.0)
    else:
        acc = u0 < e
    S[:, 0, alpha, z, y, x] = np.where(acc, -si, si).astype(S.dtype)


@pytest.mark.parametrize("name", ["ising_square4", "ising_square4_barker", "ising_sc5_odd", "ising_sc_j1j2_field",
                                  "ising_masked_field_barker", "ising_square8", "w5_ising_sc8"])
def test_host_acceptance_table_reproduces_reference_chain(name):
    """The Ising table the host builds, read through the kernels' integer key, reproduces the reference's
    recorded chain bit for bit (the GPU kernels do exactly this lookup)."""
    if not (GOLD / f"{name}.npz").exists():
        pytest.skip("fixture not generated")
    case = C.CASES[name]
    g = dict(np.load(GOLD / f"{name}.npz"))
    s = case["build"](sy, cr)
    beta = (np.float32(1.0) / g["T"]).astype(np.float32)
    keys = max(P.ising_keys(s, a) for a in range(s.b))
    table = P.ising_table(s, beta, keys)
    S = g["S0"].astype(np.int8).copy()
    for k in range(case["sweeps"]):
        for c, a in P.sweep_classes(s):
            _emulate_ising_class(s, S, table, keys, case["seed"], k, c, a)
        assert np.array_equal(S, g["snaps"][k]), f"sweep {k + 1}"


def test_bitwise_tables_match_reference_values():
    g = dict(np.load(GOLD / "tables.npz"))
    s = sy.ising("square", 4)
    for acc in ("metropolis", "barker"):
        s.acceptance = acc
        assert np.array_equal(P.p_table(s, g["betas"]), g[f"square_{acc}_p"])
        assert np.array_equal(P.p_fixed(s, g["betas"]), g[f"square_{acc}_P"])


def test_sampler_refusals_on_the_host():
    from spin_colour_kernel_b200.sampler import Sampler
    with pytest.raises(ValueError, match="Ising"):
        Sampler(sy.heisenberg("sc", 4), 32, device="cuda", bitwise=True)
    with pytest.raises(ValueError, match="bitwise"):
        Sampler(sy.ising("square", 8), 32, device="cuda", independent=True)
    with pytest.raises(ValueError, match="power of two"):
        Sampler(sy.xy("square", 8), 1, device="cuda", max_block=24)
    with pytest.raises(ValueError, match="Philox"):
        Sampler(sy.ising("sc", 128), 1024, device="cuda", bitwise=True)
    with pytest.raises(RuntimeError, match="CUDA"):
        Sampler(sy.ising("square", 4), 2, device="cpu")


def test_reference_launch_geometry_attributes():
    from spin_colour_kernel_b200.sampler import Sampler

    def geo(s, B, **kw):
        try:
            return Sampler(s, B, device="cpu", **kw)
        except RuntimeError as e:           # geometry is computed before the device is checked
            raise AssertionError(e)

    odd = sy.System("Ising sc odd periodic", 1, cr.make("sc"), (5, 5, 5), (True,) * 3, {1: 1.0})
    with pytest.raises(RuntimeError):
        Sampler(odd, 1, device="cpu")
    import spin_colour_kernel_b200.sampler as sm
    A = sm.Sampler.__new__(sm.Sampler)
    A.bitwise = False
    A.packed = False
    A.nrows = 25
    A._geometry(odd, True, None, None, 1024)
    assert (A.stride, A.bx, A.rows_per) == (5, 1, 25)
    assert odd.colouring.n_colours == 5 and sm.x_period(odd.colouring) == 5
    longrows = sy.System("Ising sc long rows", 1, cr.make("sc"), (325, 5, 1), (True, True, False), {1: 1.0})
    A.packed = True
    A.nrows = 5
    A._geometry(longrows, True, None, None, 1024)
    assert (A.stride, A.bx, A.rows_per, A.pchunks) == (5, 65, 1, 2)


def test_colouring_counts_and_clique_numbers():
    expected = {("square", (1,)): (2, 2), ("sc", (1,)): (2, 2), ("sc", (1, 2)): (4, 4), ("sc", (1, 2, 3, 4)): (9, 8),
                ("bcc", (1,)): (2, 2), ("fcc", (1,)): (4, 4), ("triangular", (1,)): (3, 3),
                ("honeycomb", (1,)): (2, 2), ("kagome", (1,)): (3, 3)}
    for key, want in expected.items():
        c = cr.make(*key)
        col = co.search(c)
        assert co.admissible(col, c)
        assert (col.n_colours, co.clique_number(c)) == want
    assert [len(cr.make(n).bonds) for n in ("square", "sc", "bcc", "fcc", "triangular", "kagome")] == \
        [4, 6, 16, 48, 6, 12]


def test_seam_condition_rejects_odd_box():
    c = cr.make("triangular")
    col = co.search(c)
    assert not co.seam_ok(col, (4, 4), (True, True))
    with pytest.raises(ValueError):
        sy.System("bad", 1, c, (4, 4), (True, True), {1: 1.0}, colouring=col)


def test_temperature_ladder_and_runner_fixture():
    """The ladder of the one-state runner, and the recorded outputs of the reference's runner it is tested on."""
    from spin_colour_kernel_b200.simulate import temperature_ladder
    assert list(temperature_ladder(2.0, 1.0, 0.5)) == [2.0, 1.5, 1.0]
    assert list(temperature_ladder(3.0, 2.0, 0.3)) == [3.0, 2.7, 2.4, 2.1]
    for bad in ((1.0, 2.0, 0.5), (2.0, 0.0, 0.5), (2.0, 1.0, 0.0)):
        with pytest.raises(ValueError):
            temperature_ladder(*bad)
    g = np.load(GOLD / "simulate.npz")
    for key, B, nT, sites in (("square", 4, 3, 64), ("sc_word", 32, 2, 64)):
        assert g[f"{key}_E"].shape == (B, nT) and g[f"{key}_M"].shape == (B, nT, 3)
        assert np.all(g[f"{key}_E2"] >= g[f"{key}_E"] ** 2 - 1e-9)        # a variance is not negative
        assert np.all(np.isin(g[f"{key}_configs"][..., 0], (-1.0, 1.0)))
        assert g[f"{key}_configs"].shape[2] == sites


def test_measure_step_and_charge_entry_points_refuse_bad_arguments_before_any_launch():
    """sck_observables_accumulate and sck_topological_charge check their arguments on the host: no device is
    touched for these refusals."""
    lib = L.lib()

    def plan_of(s, B):
        h = ctypes.c_void_p()
        L.check(lib.sck_plan_create(ctypes.byref(P.describe(s)), B, L.MODE_F32, ctypes.byref(h)))
        return h

    heis, xy = plan_of(sy.heisenberg("sc", 4), 3), plan_of(sy.xy("square", 8), 3)
    try:
        buf = L.Buffers(1, 0, 0, 1, 0, 1)
        Q = ctypes.c_void_p(1)
        assert lib.sck_topological_charge(xy, ctypes.byref(buf), Q, 3, 0, Q, None) == L.ERR_INVALID
        assert "Heisenberg" in lib.sck_last_error().decode()
        assert lib.sck_topological_charge(heis, ctypes.byref(buf), Q, 3, 4, Q, None) == L.ERR_INVALID
        assert "layer" in lib.sck_last_error().decode()
        assert lib.sck_topological_charge(heis, ctypes.byref(buf), Q, 4, 0, Q, None) == L.ERR_INVALID
        assert lib.sck_topological_charge(heis, ctypes.byref(buf), None, 3, 0, Q, None) == L.ERR_INVALID
        p = ctypes.c_void_p(1)
        assert lib.sck_observables_accumulate(heis, ctypes.byref(buf), p, L.MODE_F32, 3, 64.0, None, p, p, p, p, p,
                                              None) == L.ERR_INVALID
        assert lib.sck_observables_accumulate(heis, ctypes.byref(buf), p, L.MODE_F32, 3, 0.0, p, p, p, p, p, p,
                                              None) == L.ERR_INVALID
        assert "n_active" in lib.sck_last_error().decode()
    finally:
        lib.sck_plan_destroy(heis)
        lib.sck_plan_destroy(xy)
