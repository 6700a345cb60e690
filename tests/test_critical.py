"""The critical-point numerics (the reference's E4 pipeline) against the reference's own outputs, recorded in
`tests/golden/critical.npz` by `make_golden.py critical`: multi-histogram reweighting (with and without bootstrap
weights), Binder curves, crossings and temperature placement on the CPU; on the GPU the plain-chain series of an
Ising size, whose chain is bit-exact on every backend."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from spin_colour_kernel_b200 import critical as CR
from spin_colour_kernel_b200 import system as sy

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "critical.npz")


def test_multi_histogram_matches_the_reference():
    (a1, a2), lnZ = CR.multi_histogram(GOLD["mh_E"], [GOLD["mh_o1"], GOLD["mh_o2"]], GOLD["mh_T"], GOLD["mh_grid"],
                                       return_lnZ=True)
    np.testing.assert_allclose(lnZ, GOLD["mh_lnZ"], rtol=1e-9, atol=1e-8)
    np.testing.assert_allclose(a1, GOLD["mh_a1"], rtol=1e-9)
    np.testing.assert_allclose(a2, GOLD["mh_a2"], rtol=1e-9)
    (b1,) = CR.multi_histogram(GOLD["mh_E"], [GOLD["mh_o1"]], GOLD["mh_T"], GOLD["mh_grid"], weights=GOLD["mh_w"])
    np.testing.assert_allclose(b1, GOLD["mh_b1"], rtol=1e-9)
    # a simulated temperature reweights onto itself: the plain sample mean of its own samples
    (self_avg,) = CR.multi_histogram(GOLD["mh_E"][:1], [GOLD["mh_o1"][:1]], GOLD["mh_T"][:1], GOLD["mh_T"][:1])
    np.testing.assert_allclose(self_avg, GOLD["mh_o1"][0].mean(), rtol=1e-12)


def test_binder_crossing_and_temperatures_match_the_reference():
    U, lnZ = CR.binder_curve(GOLD["mh_E"], GOLD["mh_o1"], GOLD["mh_o2"], GOLD["mh_T"], GOLD["mh_grid"])
    np.testing.assert_allclose(U, GOLD["binder_U"], rtol=1e-9)
    np.testing.assert_allclose(lnZ, GOLD["binder_lnZ"], rtol=1e-9, atol=1e-8)
    x = np.linspace(0.0, 1.0, 9)
    got = [CR.crossing(x, np.sin(3 * x), np.cos(3 * x) * 0.5), CR.crossing(x, x, x + 1.0)]
    np.testing.assert_allclose(got, GOLD["cross"], rtol=1e-15)
    np.testing.assert_allclose(CR.e4_temperatures(4.5115, 30.0, 9, 0.05), GOLD["temps_e4"], rtol=1e-15)
    np.testing.assert_allclose(CR.e4_temperatures(4.5115, 300.0, 9, 0.01), GOLD["temps_e4_cap"], rtol=1e-15)
    assert len(CR.e4_systems()) == 8


@pytest.mark.gpu
def test_series_of_an_ising_size_matches_the_reference():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    E, m2, m4 = CR.series(sy.ising("square", 8), 8, np.array([2.1, 2.269, 2.45]), 3, 20, 12, 2, device="cuda",
                          graphs=False)
    assert np.array_equal(E, GOLD["series_E"])
    np.testing.assert_allclose(m2, GOLD["series_m2"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(m4, GOLD["series_m4"], rtol=1e-15, atol=0)
    # with graphs the chain gains the capture's warm-up sweep; the series keeps its shape and range
    E2, m22, _ = CR.series(sy.ising("square", 8), 8, np.array([2.1, 2.269, 2.45]), 3, 20, 12, 2, device="cuda")
    assert E2.shape == E.shape and np.all((m22 >= 0) & (m22 <= 1))


def test_holm_adjustment():
    """Holm's step-down adjustment: each p times the hypotheses not yet rejected, monotone, capped at 1."""
    assert np.allclose(CR.holm([0.01, 0.04, 0.03]), [0.03, 0.06, 0.06])
    assert np.allclose(CR.holm([0.5, 0.9]), [1.0, 1.0])
    assert np.allclose(CR.holm([0.001]), [0.001])


def test_crossing_estimate_extrapolates_pair_crossings():
    """On synthetic series whose reweighted Binder curves cross, the estimate is the intercept of the pair
    crossings against sqrt(L1 L2)^-x (three sizes, two pairs), and a single pair gives its own crossing."""
    rng = np.random.default_rng(0)
    temps = np.linspace(2.2, 2.34, 5)
    data = {}
    for L in (8, 16, 32):
        E = rng.normal(-1.5 * L * L, 0.5 * L, size=(5, 3, 200))
        m2 = np.abs(rng.normal(0.5, 0.05, size=(5, 3, 200)))
        m4 = m2 ** 2 * (1.0 + 0.1 * (np.arange(5)[:, None, None] - 2) * (L / 16.0))
        data[L] = {"E": E, "m2": m2, "m4": m4, "temps": temps}
    est, cross, curves = CR.crossing_estimate(data, 2.0)
    assert len(curves) == 2
    if len(cross) >= 2:
        X = np.array([l ** -2.0 for l, _ in cross])
        Y = np.array([t for _, t in cross])
        assert est == pytest.approx(float(np.polyfit(X, Y, 1)[1]))
    one = {16: data[16], 32: data[32]}
    e1, c1, _ = CR.crossing_estimate(one, 2.0)
    assert (np.isnan(e1) and not c1) or e1 == pytest.approx(c1[-1][1])


@pytest.mark.gpu
def test_e4_driver_runs_a_small_study(tmp_path):
    """The multi-size driver end to end on two small square Ising sizes: probes, series files, crossings, the
    bootstrap interval, Holm's adjustment and a verdict, written to <tag>.json."""
    import json
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = CR.e4(tmp_path, sizes2d=(8, 16), seeds=4, meas=600, boots=40, only=("Ising square",), probe_cap=2000,
                probe_start=500, tag="E4small", log=lambda *_: None)
    assert (tmp_path / "E4small.json").exists()
    assert json.loads((tmp_path / "E4small.json").read_text())["rows"][0]["system"] == "Ising square"
    assert sorted(p.name for p in tmp_path.glob("E4small-*.npz")) == ["E4small-Ising_square-L16.npz",
                                                                     "E4small-Ising_square-L8.npz"]
    r = out["rows"][0]
    assert r["sizes"] == [8, 16] and r["verdict"] in ("supported", "not supported", "inconclusive")
    assert 0.0 <= r["p_holm"] <= 1.0
    assert np.isfinite(r["estimate"]) and abs(r["estimate"] / r["T_ref"] - 1) < 0.05, r["estimate"]
    d = np.load(tmp_path / "E4small-Ising_square-L16.npz")
    assert d["E"].shape[:2] == (9, 4) and len(d["temps"]) == 9
