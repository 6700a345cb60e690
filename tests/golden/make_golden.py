"""Generate the golden fixtures by running the reference itself (its CPU path, the Triton interpreter).

Run in the development container, where the reference source is readable:

    TRITON_INTERPRET=1 python tests/golden/make_golden.py [--ref /root/reference/src] [case ...]

Writes one `<case>.npz` per parity case of cases.py (initial spins, spins after recorded sweeps, energies and
magnetizations per sweep, the temperatures, the acceptance tables of bitwise cases) plus `philox.npz`
(Triton's own rand4x / randint4x outputs) and `quickstart.json`. Nothing on the GPU side reads the
reference: the fixtures are the committed record of its outputs.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

os.environ.setdefault("TRITON_INTERPRET", "1")
HERE = Path(__file__).resolve().parent


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference/src")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args(argv)
    os.environ.setdefault("SCK_CACHE", str(Path("/tmp") / "sck_golden_cache"))
    sys.path.insert(0, a.ref)
    sys.path.insert(0, str(HERE))
    import numpy as np
    import torch
    from Spin_Colour_Kernel import bitwise as bw
    from Spin_Colour_Kernel import crystals as cr
    from Spin_Colour_Kernel import system as sy
    from Spin_Colour_Kernel.sampler import Sampler

    import cases as C

    names = a.cases or list(C.CASES) + ["philox", "quickstart", "tables", "simulate", "runs", "anneal", "critical"]
    for name in names:
        t0 = time.time()
        if name == "philox":
            _philox(np, torch, bw)
        elif name == "quickstart":
            _quickstart(torch, sy, Sampler)
        elif name == "tables":
            _tables(np, bw, sy, cr)
        elif name == "simulate":
            _simulate(np, a.ref)
        elif name == "runs":
            _runs(np, sy)
        elif name == "anneal":
            _anneal(np, torch, sy, Sampler)
        elif name == "critical":
            _critical(np, sy)
        else:
            case = C.CASES[name]
            s = case["build"](sy, cr)
            kw = C.sampler_kwargs(case)
            if case.get("ref_packed") is not None:
                kw["packed"] = case["ref_packed"]
            B = case["B"]
            A = Sampler(s, B, device="cpu", seed=case["seed"], **kw)
            T = C.temperatures(case["T"], B)
            A.set_temperature(torch.from_numpy(T))
            S = A.init_spins(seed=case["init"])
            rec = {"T": T, "S0": A.unpack(S).numpy().copy(), "E": [], "M": [], "ptab": []}
            if A.packed:
                rec["W0"] = S.numpy().copy()
            every = case.get("record_every", 1)
            keep = set(range(1, case["sweeps"] + 1)) if every else {1, 2, 10, 50, 100, case["sweeps"]}
            if A.bitwise:
                rec["ptab"] = A.ptab.numpy().copy()
            snaps, snap_ids = [], []
            for k in range(1, case["sweeps"] + 1):
                A.sweep(S)
                x = A.unpack(S)
                rec["E"].append(A.energy(S).numpy().copy())
                rec["M"].append(A.magnetization(S).numpy().copy())
                if k in keep:
                    snaps.append(x.numpy().copy())
                    snap_ids.append(k)
            out = dict(T=rec["T"], S0=rec["S0"], E=np.stack(rec["E"]), M=np.stack(rec["M"]),
                       snaps=np.stack(snaps), snap_ids=np.asarray(snap_ids), n_colours=s.colouring.n_colours,
                       classes=np.asarray(A.classes, np.int64), stride=A.stride, bx=A.bx, rows_per=A.rows_per)
            if A.packed:
                out["W0"] = rec["W0"]
                out["Wend"] = S.numpy().copy()
            if A.bitwise:
                out["ptab"] = rec["ptab"]
            np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"{name}: {time.time() - t0:.1f} s", flush=True)


def _philox(np, torch, bw):
    import triton
    import triton.language as tl

    @triton.jit
    def k4(out_ptr, seed, N: tl.constexpr):
        off = tl.arange(0, N)
        a, b, c, d = tl.rand4x(seed, off * 7919 + 3)
        tl.store(out_ptr + off, a)
        tl.store(out_ptr + N + off, b)
        tl.store(out_ptr + 2 * N + off, c)
        tl.store(out_ptr + 3 * N + off, d)

    @triton.jit
    def ki(out_ptr, seed, N: tl.constexpr):
        off = tl.arange(0, N)
        a, b, c, d = tl.randint4x(seed, off * 104729 + 11)
        tl.store(out_ptr + off, a.to(tl.int32, bitcast=True))
        tl.store(out_ptr + N + off, b.to(tl.int32, bitcast=True))
        tl.store(out_ptr + 2 * N + off, c.to(tl.int32, bitcast=True))
        tl.store(out_ptr + 3 * N + off, d.to(tl.int32, bitcast=True))

    seeds = [0, 1, 12345, 123457, 2147483628, bw.sweep_seed(1234, 0), bw.sweep_seed(1234, 199)]
    N = 256
    U, R = [], []
    for sd in seeds:
        out = torch.zeros(4 * N)
        k4[(1,)](out, sd, N=N)
        U.append(out.numpy().reshape(4, N).copy())
        outi = torch.zeros(4 * N, dtype=torch.int32)
        ki[(1,)](outi, sd, N=N)
        R.append(outi.numpy().view(np.uint32).reshape(4, N).copy())
    np.savez_compressed(HERE / "philox.npz", seeds=np.asarray(seeds, np.int64), N=N, rand4x=np.stack(U),
                        randint4x=np.stack(R), offset_mul=7919, offset_add=3, int_mul=104729, int_add=11,
                        sweep_seeds=np.asarray([[bw.sweep_seed(b, s) for s in range(0, 50)] for b in (0, 1, 1234, 99991)]))


def _quickstart(torch, sy, Sampler):
    """The reference's quick start: 3 systems, 2 replicas, seed 11, T = 1.5, init seed 2, 20 sweeps."""
    rows = []
    for s in [sy.ising("square", 8), sy.xy("sc", 4), sy.heisenberg("triangular", 6)]:
        A = Sampler(s, 2, device="cpu", seed=11)
        A.set_temperature(1.5)
        S = A.init_spins(seed=2)
        A.sweep(S, 20)
        e = (A.energy(S).double() / s.n_active).tolist()
        rows.append(dict(name=s.name, colours=s.colouring.n_colours, energy_per_site=e))
    (HERE / "quickstart.json").write_text(json.dumps(rows, indent=1))


def _tables(np, bw, sy, cr):
    betas = np.array([0.25, 0.5, 1.0 / 2.269, 1.0 / 4.5115, 2.0])
    out = {}
    for key, s in {"square": sy.ising("square", 4), "sc": sy.ising("sc", 4), "fcc": sy.ising("fcc", 4),
                   "triangular": sy.ising("triangular", 6)}.items():
        for acc in ("metropolis", "barker"):
            s.acceptance = acc
            out[f"{key}_{acc}_p"] = bw.p_table(s, betas)
            out[f"{key}_{acc}_P"] = bw.p_fixed(s, betas)
    m = sy.System("masked h", 1, cr.make("square"), (8, 8), (True, True), {1: 1.0}, h=(0.3,),
                  mask=np.random.default_rng(0).random((1, 1, 8, 8)) > 0.25)
    out["masked_h_metropolis_p"] = bw.p_table(m, betas)
    out["masked_h_metropolis_P"] = bw.p_fixed(m, betas)
    out["betas"] = betas
    np.savez_compressed(HERE / "tables.npz", **out)


def _simulate(np, ref):
    """The reference's one-state ladder runner (simulate.py:322-402) on its CPU path: Ising chains (bit-exact on
    every backend), so the accumulated FP64 observables are a fixture for the same runner on the GPU."""
    from Spin_Colour_Kernel import simulate as SIM
    out = {}
    runs = {
        "square": (SIM.build_system("ising", "square", (8, 8), (True, True), {"J": {1: 1.0}, "H": 0.1}),
                   dict(replicas=4, temps=[3.0, 2.5, 2.0], n_therm=4, n_meas=6, every=2, config_every=2, seed=1)),
        "sc_word": (SIM.build_system("ising", "sc", (4, 4, 4), (True, True, True), {"J": {1: 1.0}}),
                    dict(replicas=32, temps=[5.0, 4.0], n_therm=3, n_meas=4, every=1, config_every=1, seed=2)),
    }
    for key, (s, kw) in runs.items():
        r = SIM.simulate_state(s, device="cpu", kB=1.0, log=lambda m: None, **kw)
        for f in ("M", "E", "E2", "Mabs", "M2", "configs", "config_temperatures"):
            out[f"{key}_{f}"] = np.asarray(r[f])
    np.savez_compressed(HERE / "simulate.npz", **out)


def _runs(np, sy):
    """The reference's run driver (simulate.py): geometry, Hamiltonians, prepared files, collect, and a small
    Ising run in two replica blocks on its CPU path."""
    import tempfile
    from Spin_Colour_Kernel import simulate as SIM
    out = {}
    import cases as C
    for i, (cry, box, coords, shape) in enumerate(C.SHAPES):
        pos, mask = SIM.active_sites(cry, box, coords, shape)
        out[f"shape{i}_pos"], out[f"shape{i}_mask"] = pos, mask
    for i, (model, cry, box, per, coords, shape, theta) in enumerate(C.THETAS):
        _, mask = SIM.active_sites(cry, box, coords, shape)
        s = SIM.build_system(model, cry, box, per, theta, mask=mask if shape else None, log=lambda m: None)
        out[f"theta{i}_bonds"] = np.stack([s.bond_matrix(k) for k in range(len(s.crystal.bonds))])
        out[f"theta{i}_k1"] = np.zeros(0) if s.cubic_k1 is None else s.cubic_k1
        out[f"theta{i}_h"] = np.zeros(0) if s.h is None else np.asarray(s.h)
        out[f"theta{i}_periodic"] = np.asarray(s.periodic)
        out[f"theta{i}_k2"] = np.float64(s.cubic_k2)
    with tempfile.TemporaryDirectory() as d:
        run = SIM.prepare(dict(C.RUN_CFG), d, log=lambda m: None)
        out["run_json"] = np.array((Path(d) / "run.json").read_text())
        out["run_sites"] = np.load(Path(d) / "sites.npy")
        out["run_mask"] = np.load(Path(d) / "mask.npy")
        for part, rng in enumerate(SIM.replica_blocks(run["replicas"], 2)):
            SIM.run(run, [0, 1], d, device="cpu", log=lambda m: None, replicas=rng, part=part)
        res = SIM.collect(d)
        for k, v in res.items():
            out[f"run_res_{k}"] = v
        out["run_configs"] = np.load(Path(d) / "configurations.npy")
        z = np.load(Path(d) / "state_001_p01.npz")
        out["run_state_keys"] = np.array(sorted(z.files))
    np.savez_compressed(HERE / "runs.npz", **out)


def _anneal(np, torch, sy, Sampler):
    """The reference's nanodisk observer (E, mean magnetization vector, middle-layer charge; anneal.py:83-146)
    on states after a few low-temperature sweeps, its reducer on a fixed accumulator array, and its helpers."""
    from Spin_Colour_Kernel import anneal as AN
    out = {}
    for i, (params, Rd, L, angle, shells) in enumerate(
            [((0.0, 0.0, 0.0, 0.177, 0.139, 0.483, 0.88), 3.3, 3, 90.0, (1,)),
             ((0.2, 0.0, 0.0, 0.1, 0.2, 0.3, 1.2), 4.2, 3, 30.0, (1, 2))]):
        s = AN.build_state(params, Rd, L, angle, shells)
        A = Sampler(s, 3, "cpu", 7)
        A.set_temperature(0.05)
        S = A.init_spins(seed=5)
        A.sweep(S, 6)
        E, Mv, Q = AN.Observer(A)(S)
        out[f"state{i}_S"] = S.numpy().copy()
        out[f"state{i}_E"], out[f"state{i}_Mv"], out[f"state{i}_Q"] = E.numpy(), Mv.numpy(), Q.numpy()
        out[f"state{i}_k1"] = s.cubic_k1
        out[f"state{i}_bonds"] = np.stack([s.bond_matrix(k) for k in range(len(s.crystal.bonds))])
    rng = np.random.default_rng(3)
    obs = rng.normal(size=(4, 8, 5))
    obs[:, 1] = obs[:, 0] ** 2 + rng.random((4, 5))
    obs[:, 3] = obs[:, 2] ** 2 + rng.random((4, 5))
    temps = np.array([40.0, 30.0, 20.0, 10.0])
    out["reduce_obs"], out["reduce_T"] = obs, temps
    for k, v in AN.reduce_obs(obs, temps, 221).items():
        out[f"reduce_{k}_out"] = v
    out["shells"] = np.asarray(AN.active_shells([[0.0, 0.1, 0.0, 1, 1, 1, 1], [0.0, 0.0, 0.2, 1, 1, 1, 1]]))
    np.savez_compressed(HERE / "anneal.npz", **out)


def _critical(np, sy):
    """The reference's E4 numerics (exp_perf.py:728-822): the series of plain chains on its CPU path (an Ising
    size, bit-exact everywhere), multi-histogram reweighting, Binder curves and their crossing."""
    from Spin_Colour_Kernel import exp_perf as EP
    out = {}
    s = sy.ising("square", 8)
    temps = np.array([2.1, 2.269, 2.45])
    E, m2, m4 = EP._series(s, 8, temps, 3, 20, 12, 2, "cpu")
    out["series_E"], out["series_m2"], out["series_m4"] = E, m2, m4
    rng = np.random.default_rng(11)
    T = np.array([1.9, 2.0, 2.1, 2.2, 2.3])
    Es = np.stack([rng.normal(-200 + 40 * t, 8.0, 400) for t in T])          # overlapping energy histograms
    o1 = np.tanh(-Es / 100.0) ** 2
    o2 = o1 ** 2
    grid = np.linspace(1.95, 2.25, 7)
    (a1, a2), lnZ = EP.multi_histogram(Es, [o1, o2], T, grid, return_lnZ=True)
    wts = rng.integers(0, 3, size=Es.shape).astype(np.float64)
    (b1,) = EP.multi_histogram(Es, [o1], T, grid, weights=wts)
    U, lnZb = EP._binder_curve(Es, o1, o2, T, grid)
    out.update(mh_E=Es, mh_o1=o1, mh_o2=o2, mh_T=T, mh_grid=grid, mh_a1=a1, mh_a2=a2, mh_lnZ=lnZ, mh_w=wts,
               mh_b1=b1, binder_U=U, binder_lnZ=lnZb)
    x = np.linspace(0.0, 1.0, 9)
    out["cross"] = np.array([EP._crossing(x, np.sin(3 * x), np.cos(3 * x) * 0.5), EP._crossing(x, x, x + 1.0)])
    out["temps_e4"] = EP.e4_temperatures(4.5115, 30.0, 9, 0.05)
    out["temps_e4_cap"] = EP.e4_temperatures(4.5115, 300.0, 9, 0.01)
    np.savez_compressed(HERE / "critical.npz", **out)


if __name__ == "__main__":
    main()
