"""The nanodisk cooling ladder (the reference's `anneal` module) against the reference's own outputs, recorded in
`tests/golden/anneal.npz` by `make_golden.py anneal`: the nanodisk Hamiltonians, the reducer, the shells
helper and the FP64 host restatement of the Berg-Luscher charge on the CPU; on the GPU the observer (library
observables pass plus the charge kernel) on the reference's own states, and a short ladder."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import observables as obs
from spin_colour_kernel_b200 import anneal as AN

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "anneal.npz")
STATES = [((0.0, 0.0, 0.0, 0.177, 0.139, 0.483, 0.88), 3.3, 3, 90.0, (1,)),
          ((0.2, 0.0, 0.0, 0.1, 0.2, 0.3, 1.2), 4.2, 3, 30.0, (1, 2))]


@pytest.mark.parametrize("i", range(len(STATES)))
def test_nanodisk_states_match_the_reference(i):
    s = AN.build_state(*STATES[i])
    bonds = np.stack([s.bond_matrix(k) for k in range(len(s.crystal.bonds))])
    np.testing.assert_allclose(bonds, GOLD[f"state{i}_bonds"], rtol=0, atol=1e-15)
    assert np.array_equal(s.cubic_k1, GOLD[f"state{i}_k1"])


@pytest.mark.parametrize("i", range(len(STATES)))
def test_host_charge_restatement_matches_the_reference(i):
    s = AN.build_state(*STATES[i])
    mid = s.L3 // 2
    S = GOLD[f"state{i}_S"].astype(np.float64)
    disk = s.site_mask()[0, mid]
    valid = (disk[:-1, :-1] & disk[:-1, 1:] & disk[1:, :-1] & disk[1:, 1:]).astype(np.float64)
    np.testing.assert_allclose(obs.berg_luscher_q(S[:, :, 0, mid], valid), GOLD[f"state{i}_Q"], rtol=1e-12,
                               atol=1e-13)


def test_reducer_and_shells_match_the_reference():
    got = AN.reduce_obs(GOLD["reduce_obs"], GOLD["reduce_T"], 221)
    for k, v in got.items():
        np.testing.assert_allclose(v, GOLD[f"reduce_{k}_out"], rtol=1e-14, atol=0, err_msg=k)
    assert AN.active_shells([[0.0, 0.1, 0.0, 1, 1, 1, 1], [0.0, 0.0, 0.2, 1, 1, 1, 1]]) == GOLD["shells"].tolist()
    with pytest.raises(ValueError):
        AN.reduce_obs(np.zeros((3, 7, 2)), [1.0, 2.0, 3.0], 10)


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(STATES)))
def test_observer_on_the_references_states(i):
    """E, the mean magnetization vector and the middle-layer charge of the reference's own spins: library FP64
    observables and the charge kernel against the reference's torch FP64 observer."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spin_colour_kernel_b200.sampler import Sampler
    s = AN.build_state(*STATES[i])
    S = torch.from_numpy(GOLD[f"state{i}_S"]).cuda().contiguous()
    A = Sampler(s, S.shape[0], "cuda", 7)
    E, Mv, Q = AN.Observer(A)(S)
    np.testing.assert_allclose(E.cpu().numpy(), GOLD[f"state{i}_E"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(Mv.cpu().numpy(), GOLD[f"state{i}_Mv"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(Q.cpu().numpy(), GOLD[f"state{i}_Q"], rtol=1e-12, atol=1e-13)


@pytest.mark.gpu
def test_a_short_ladder_runs_with_graphs():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    s = AN.build_state(*STATES[0])
    assert isinstance(AN.check_exact(s, "cuda"), int)      # the count itself depends on the float32 path
    temps = np.array([40.0, 20.0, 5.0])
    r = AN.anneal_state(s, 4, temps, n_therm=20, n_meas=10, every=2, seed=3, device="cuda", log=lambda m: None)
    assert r["obs"].shape == (3, 8, 4) and r["mvec"].shape == (3, 4, 3) and r["snaps"].shape == (3, 9, 9)
    assert np.all(np.isfinite(r["obs"])) and np.all(r["obs"][:, 1] >= r["obs"][:, 0] ** 2 - 1e-9)
    red = AN.reduce_obs(r["obs"], temps, s.n_active)
    assert np.all(red["M"] <= 1 + 1e-9) and red["Q"].shape == (3,)
