"""The run driver (the reference's `simulate.py` prepare / run / collect, its geometry and Hamiltonian builder)
against the reference's own outputs, recorded in `tests/golden/runs.npz` by `make_golden.py runs`.

CPU: active-site masks and positions, built Hamiltonians (bond matrices with DMI, surface anisotropy, fields,
the fallback to open boundaries), the prepared files byte for byte, `collect`'s combined arrays, and the refusals
of shapes that are not conditions on the coordinates. GPU: a prepared two-state Ising run in two replica blocks
(bit-exact chains) gives the reference's results and configurations.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import cases as C
from spin_colour_kernel_b200 import simulate as SIM

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "runs.npz")


@pytest.mark.parametrize("i", range(len(C.SHAPES)))
def test_active_sites_match_the_reference(i):
    cry, box, coords, shape = C.SHAPES[i]
    pos, mask = SIM.active_sites(cry, box, coords, shape)
    np.testing.assert_allclose(pos, GOLD[f"shape{i}_pos"], rtol=0, atol=1e-12)
    assert np.array_equal(mask, GOLD[f"shape{i}_mask"])


@pytest.mark.parametrize("i", range(len(C.THETAS)))
def test_built_hamiltonians_match_the_reference(i):
    model, cry, box, per, coords, shape, theta = C.THETAS[i]
    _, mask = SIM.active_sites(cry, box, coords, shape)
    s = SIM.build_system(model, cry, box, per, theta, mask=mask if shape else None, log=lambda m: None)
    bonds = np.stack([s.bond_matrix(k) for k in range(len(s.crystal.bonds))])
    np.testing.assert_allclose(bonds, GOLD[f"theta{i}_bonds"], rtol=0, atol=1e-15)
    k1 = np.zeros(0) if s.cubic_k1 is None else s.cubic_k1
    assert np.array_equal(k1, GOLD[f"theta{i}_k1"])
    h = np.zeros(0) if s.h is None else np.asarray(s.h)
    np.testing.assert_allclose(h, GOLD[f"theta{i}_h"], rtol=0, atol=1e-15)
    assert tuple(s.periodic) == tuple(GOLD[f"theta{i}_periodic"])
    assert s.cubic_k2 == float(GOLD[f"theta{i}_k2"])


def test_prepared_files_are_the_references(tmp_path):
    run = SIM.prepare(dict(C.RUN_CFG), tmp_path, log=lambda m: None)
    assert (tmp_path / "run.json").read_text() == str(GOLD["run_json"])
    assert np.array_equal(np.load(tmp_path / "sites.npy"), GOLD["run_sites"])
    assert np.array_equal(np.load(tmp_path / "mask.npy"), GOLD["run_mask"])
    cf = np.load(tmp_path / "configurations.npy", mmap_mode="r")
    assert cf.shape == GOLD["run_configs"].shape and cf.dtype == np.float32
    assert run["n_sites"] == int(GOLD["run_mask"].sum())


def test_collect_combines_blocks_as_the_reference_does(tmp_path):
    """State files cut from the reference's combined arrays (two blocks per state) collect back to them, with
    the reference's Cv, chi and per-site means."""
    run = SIM.prepare(dict(C.RUN_CFG), tmp_path, log=lambda m: None)
    res = {k[len("run_res_"):]: GOLD[k] for k in GOLD.files if k.startswith("run_res_")}
    for i in range(len(run["states"])):
        for part, (r0, r1) in enumerate(SIM.replica_blocks(run["replicas"], 2)):
            np.savez(tmp_path / f"state_{i:03d}_p{part:02d}.npz", r0=r0, r1=r1, M=res["magnetization"][i, r0:r1],
                     E=res["energy"][i, r0:r1], E2=res["energy2"][i, r0:r1], Mabs=res["Mabs"][i, r0:r1],
                     M2=res["M2"][i, r0:r1], config_temperatures=np.asarray(run["config_temperatures"]))
    got = SIM.collect(tmp_path)
    assert sorted(got) == sorted(res)
    for k, v in res.items():
        if v.dtype.kind in "US":
            assert np.array_equal(got[k], v), k
        else:
            np.testing.assert_allclose(got[k], v, rtol=1e-14, atol=0, err_msg=k)
    z = np.load(tmp_path / "results.npz")
    assert sorted(z.files) == sorted(res)
    assert np.array_equal(np.load(tmp_path / "magnetization.npy"), res["magnetization"])


def test_collect_refuses_a_missing_block(tmp_path):
    run = SIM.prepare(dict(C.RUN_CFG), tmp_path, log=lambda m: None)
    for i in range(len(run["states"])):
        z = {k: np.zeros((2, 3)) for k in ("E", "E2", "Mabs", "M2")}
        np.savez(tmp_path / f"state_{i:03d}_p00.npz", r0=0, r1=2, M=np.zeros((2, 3, 3)), **z)
    with pytest.raises(ValueError, match="replicas"):
        SIM.collect(tmp_path)


def test_replica_blocks_sizes_and_estimate():
    assert SIM.replica_blocks(10, 4) == [(0, 3), (3, 6), (6, 8), (8, 10)]
    assert SIM.replica_blocks(32, 2) == [(0, 16), (16, 32)]
    assert SIM.replica_blocks(3, 8) == [(0, 1), (1, 2), (2, 3)]
    assert abs(SIM.size_estimate_gb(2, 128, 200, 5000) - 2 * 128 * 200 * 5000 * 12 / 1e9) < 1e-12


@pytest.mark.parametrize("shape", ["().__class__.__bases__[0].__subclasses__()", "__import__('os').system('true')",
                                   "(lambda: 1)()", "x.real <= 2", "'a' < 'b'", "open('f')", "abs(x, key=1) < 2",
                                   "(x < 1) and (y < 1)", "q < 1"])
def test_a_shape_that_is_not_a_condition_on_the_coordinates_is_refused(shape):
    with pytest.raises(ValueError):
        SIM.active_sites("sc", [4, 4, 4], "cartesian", shape)


def test_a_constant_shape_keeps_every_site_as_the_reference_does():
    _, mask = SIM.active_sites("sc", [4, 4, 4], "cartesian", "True")
    assert mask.all()


def test_shape_refusals_name_what_to_use():
    with pytest.raises(ValueError, match=r"use & \(and\)"):
        SIM.active_sites("sc", [4, 4, 4], "cartesian", "(x < 1) or (y < 1)")
    with pytest.raises(ValueError, match="cartesian"):
        SIM.active_sites("sc", (4, 4, 4), "toroidal", "r < 1")
    with pytest.raises(ValueError, match="coordinate"):
        SIM.active_sites("sc", (4, 4, 4), "", "r < 1")
    with pytest.raises(ValueError, match="no site"):
        SIM.active_sites("sc", (4, 4, 4), "spherical", "r < 0")
    with pytest.raises(ValueError, match="Heisenberg"):
        SIM.build_system("ising", "square", (8, 8), (True, True), {"J": {1: 1.0}, "D": 0.5})
    with pytest.raises(ValueError, match="unknown parameters"):
        SIM.build_system("xy", "square", (8, 8), (True, True), {"J": {1: 1.0}, "B": 0.5})


@pytest.mark.gpu
def test_a_prepared_run_in_two_blocks_gives_the_references_results(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    run = SIM.prepare(dict(C.RUN_CFG), tmp_path, log=lambda m: None)
    run = json.loads((tmp_path / "run.json").read_text())
    for part, rng in enumerate(SIM.replica_blocks(run["replicas"], 2)):
        SIM.run(run, [0, 1], tmp_path, device="cuda", log=lambda m: None, replicas=rng, part=part, graphs=False)
    got = SIM.collect(tmp_path)
    for k in ("magnetization", "energy", "energy2", "Mabs", "M2", "Cv", "chi", "E_site", "M_site"):
        np.testing.assert_allclose(got[k], GOLD[f"run_res_{k}"], rtol=1e-12, atol=1e-9, err_msg=k)
    assert np.array_equal(np.load(tmp_path / "configurations.npy"), GOLD["run_configs"])
    assert sorted(np.load(tmp_path / "state_001_p01.npz").files) == sorted(GOLD["run_state_keys"].tolist())
