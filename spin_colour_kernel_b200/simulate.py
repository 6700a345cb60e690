"""One state of a temperature ladder on the sm_100a library: the reference's `simulate.simulate_state`
(`src/Spin_Colour_Kernel/simulate.py:322-402`) with the same arguments, the same outputs and the same chain.

For each temperature (descending ladder, one chain per replica carried from one temperature to the next) the
runner thermalises, takes the FP64 energy of the state as a reference E_ref, then makes m = n_meas // every
observations, each after `every` sweeps. An observation adds, per replica, E - E_ref, (E - E_ref)^2, |m|,
|m|^2 and the mean magnetization vector m to FP64 accumulators; the results are
    E = E_ref + <E - E_ref>,  E2 = <(E - E_ref)^2> + 2 E_ref <E - E_ref> + E_ref^2,
    Mabs = <|m|>,  M2 = <|m|^2>,  M = <m> (float32, three components),
and every `config_every`-th temperature saves each replica's active-site spins.

Where the reference runs the observation as a chain of torch operations on an FP64 copy of the state
(`simulate.py:267-319`), here one library call does it: the observables pass (`sck_observables`) and a fold of
its result into the accumulators on the device (`sck_observables_accumulate`). The measure step — `every`
sweeps and that call — is captured once in a CUDA graph and replayed (packed Ising excepted, as in the
reference), and thermalisation replays a graph of 10 x `every` sweeps.
"""

from __future__ import annotations

import ast
import json
import time
from pathlib import Path

import numpy as np
import torch

from . import crystals as cr
from .sampler import Sampler
from .system import System

#: spin components per model name
MODELS = {"ising": 1, "xy": 2, "heisenberg": 3}
#: coordinate names a shape may use, per coordinate system (origin at the centre of the box, radians)
COORDS = {"cartesian": ("x", "y", "z"), "spherical": ("r", "theta", "phi"), "cylindrical": ("rho", "phi", "z")}
#: Boltzmann constant in meV / K (temperatures in kelvin when `units` is "meV")
KB_MEV = 0.086173404


def temperature_ladder(T_max: float, T_min: float, T_step: float) -> np.ndarray:
    """Descending temperatures T_max, T_max - T_step, ..., down to T_min (`simulate.py:243-249`)."""
    hi, lo, step = float(T_max), float(T_min), float(T_step)
    if step <= 0 or lo <= 0 or hi < lo:
        raise ValueError("need T_max >= T_min > 0 and T_step > 0")
    count = int(np.floor((hi - lo) / step + 1e-9)) + 1
    return np.round(hi - step * np.arange(count), 10)


def site_spins(A: Sampler, S: torch.Tensor, mask: np.ndarray) -> np.ndarray:
    """(B, n_active, 3) float32 spins of the active sites in (b, z, y, x) order; missing components are 0."""
    x = A.unpack(S).float()                                   # (B, n, b, L3, L2, L1)
    B, n = x.shape[0], x.shape[1]
    flat = x.reshape(B, n, -1)[:, :, torch.from_numpy(mask.reshape(-1)).to(x.device)]
    out = np.zeros((B, flat.shape[2], 3), np.float32)
    out[:, :, :n] = flat.permute(0, 2, 1).cpu().numpy()
    return out


class _Measure:
    """Device buffers of one state's measurements and the calls that fill them."""

    def __init__(self, A: Sampler, S: torch.Tensor):
        s, dev = A.sys, A.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.A, self.S = A, S
        self.E_ref = torch.zeros(A.B, **f64)
        self.E = torch.zeros(A.B, **f64)
        self.M = torch.zeros((A.B, s.b, s.n), **f64)
        self.acc = torch.zeros((4, A.B), **f64)
        self.accv = torch.zeros((A.B, s.n), **f64)

    def reference(self):
        self.A.observables(self.S, self.E_ref, self.M)

    def clear(self):
        self.acc.zero_()
        self.accv.zero_()

    def step(self, every: int):
        self.A.sweep(self.S, every)
        self.A.observe(self.S, self.E_ref, self.acc, self.accv, self.E, self.M)


def simulate_state(s: System, replicas: int, temps, n_therm: int, n_meas: int, every: int, config_every: int,
                   seed: int, device="cuda", kB: float = 1.0, log=print, graphs: bool | None = None) -> dict:
    """Run the ladder `temps` for one system; energies are totals, M is the mean magnetization per site.

    Returns M (B, nT, 3) float32, E, E2, Mabs, M2 (B, nT) float64, configs (B, n_saved, n_active, 3) float32 and
    config_temperatures, as the reference does. `graphs=False` replays nothing (every launch from the host)."""
    A = Sampler(s, int(replicas), device, seed)
    S = A.init_spins(seed=seed)
    mask = s.site_mask()
    every = max(1, int(every))
    n_obs = max(1, int(n_meas) // every)
    block = 10 * every
    ce = max(1, int(config_every))
    temps = np.asarray(temps, float)
    nT, B = len(temps), int(replicas)
    saved = [t for t in range(nT) if t % ce == 0]
    out = dict(M=np.zeros((B, nT, 3), np.float32), E=np.zeros((B, nT)), E2=np.zeros((B, nT)),
               Mabs=np.zeros((B, nT)), M2=np.zeros((B, nT)),
               configs=np.zeros((B, len(saved), int(mask.sum()), 3), np.float32),
               config_temperatures=temps[saved])
    meas = _Measure(A, S)
    use_graphs = (A.device.type == "cuda" and not A.packed) if graphs is None else bool(graphs)
    A.set_temperature(kB * float(temps[0]))
    if use_graphs:
        therm = A.graph(S, block)
        dev = A.device
        with torch.cuda.device(dev):
            side = torch.cuda.Stream(device=dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                meas.step(every)                          # warm-up (workspace, lazy state) outside the capture
            torch.cuda.current_stream(dev).wait_stream(side)
            torch.cuda.synchronize(dev)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                meas.step(every)

        def observe_step():
            with torch.cuda.device(dev):
                g.replay()
    else:
        def therm():
            A.sweep(S, block)

        def observe_step():
            meas.step(every)

    t0 = time.perf_counter()
    for t, T in enumerate(temps):
        A.set_temperature(kB * float(T))
        for _ in range(int(n_therm) // block):
            therm()
        if int(n_therm) % block:
            A.sweep(S, int(n_therm) % block)
        meas.reference()
        meas.clear()
        for _ in range(n_obs):
            observe_step()
        d, d2, ma, m2 = (meas.acc / n_obs).cpu().numpy()
        er = meas.E_ref.cpu().numpy()
        out["E"][:, t] = er + d
        out["E2"][:, t] = d2 + 2 * er * d + er * er
        out["Mabs"][:, t] = ma
        out["M2"][:, t] = m2
        out["M"][:, t, :s.n] = (meas.accv / n_obs).float().cpu().numpy()
        if t in saved:
            out["configs"][:, saved.index(t)] = site_spins(A, S, mask)
        if t % max(1, nT // 10) == 0 or t == nT - 1:
            log(f"    T = {T:9.4f}   <E>/site = {out['E'][:, t].mean() / s.n_active:+.4f}"
                f"   <|M|> = {out['Mabs'][:, t].mean():.4f}   {time.perf_counter() - t0:8.1f} s")
    return out


# ---------------------------------------------------------------------------------------------- geometry
# A shape is a boolean condition on coordinate arrays, written with arithmetic, comparisons, & | ^ ~ and the
# functions below (simulate.py:62-91 of the reference). It is parsed and every node checked before it is
# evaluated with no builtins, so only those names can be reached.
_FUNCS = {name: getattr(np, name) for name in ("sqrt", "sin", "cos", "tan", "arctan2", "arccos", "exp", "log",
                                               "minimum", "maximum", "mod", "floor", "ceil")}
_FUNCS["abs"] = np.abs
_CONSTS = {"pi": np.pi}
_ALLOWED = (ast.Expression, ast.BinOp, ast.UnaryOp, ast.Compare, ast.Call, ast.Name, ast.Load, ast.Constant,
            ast.Add, ast.Sub, ast.Mult, ast.Div, ast.FloorDiv, ast.Mod, ast.Pow, ast.BitAnd, ast.BitOr, ast.BitXor,
            ast.Invert, ast.USub, ast.UAdd, ast.Lt, ast.LtE, ast.Gt, ast.GtE, ast.Eq, ast.NotEq)


def _validate_shape(shape: str, coords: tuple) -> None:
    try:
        tree = ast.parse(shape, mode="eval")
    except SyntaxError as e:
        raise ValueError(f"the shape {shape!r} is not a valid condition: {e.msg}") from None
    funcs = ", ".join(sorted(_FUNCS))
    for node in ast.walk(tree):
        if isinstance(node, (ast.BoolOp, ast.Not)):
            raise ValueError("use & (and), | (or), ~ (not) in a shape, with parentheses around each comparison")
        if not isinstance(node, _ALLOWED):
            raise ValueError(f"the shape {shape!r} may hold only numbers, coordinates, operators and {funcs}; "
                             f"found {type(node).__name__}")
        if isinstance(node, ast.Constant) and not isinstance(node.value, (int, float)):
            raise ValueError(f"the shape {shape!r} may hold only numbers as constants")
        if isinstance(node, ast.Call):
            if not (isinstance(node.func, ast.Name) and node.func.id in _FUNCS) or node.keywords:
                raise ValueError(f"the shape {shape!r} calls something other than {funcs}")
        if isinstance(node, ast.Name) and node.id not in _FUNCS and node.id not in _CONSTS and node.id not in coords:
            raise ValueError(f"name {node.id!r} is not defined; the coordinates are {', '.join(coords)}")


def site_positions(crystal: cr.Crystal, box) -> np.ndarray:
    """Cartesian position (b, L3, L2, L1, 3) of every site, centred on the box (z = 0 for 2D crystals)."""
    D, b = crystal.D, crystal.b
    sizes = [int(v) for v in box] + [1] * (3 - len(box))
    L1, L2, L3 = sizes
    cz, cy, cx = np.meshgrid(np.arange(L3), np.arange(L2), np.arange(L1), indexing="ij")
    cell = np.stack((cx, cy, cz), axis=-1)[..., :D].astype(float)
    pos = np.zeros((b, L3, L2, L1, 3))
    for a in range(b):
        pos[a, ..., :D] = (cell + crystal.basis[a]) @ crystal.vectors
    return pos - pos.reshape(-1, 3).mean(axis=0)


def active_sites(crystal, box, coords: str = "", shape: str = ""):
    """(positions (b, L3, L2, L1, 3), mask (b, L3, L2, L1)) of the sites a shape keeps
    (`simulate.py:110-145`). `coords` names the coordinate system of `shape` — cartesian (x, y, z), spherical
    (r, theta, phi) or cylindrical (rho, phi, z), origin at the box centre, radians; e.g. "r <= 10" or
    "(rho <= 8) & (abs(z) <= 2)". An empty shape keeps every site."""
    c = crystal if isinstance(crystal, cr.Crystal) else cr.make(str(crystal))
    if len(box) != c.D:
        raise ValueError(f"crystal {c.name} needs a box of {c.D} sizes, got {list(box)}")
    pos = site_positions(c, box)
    system, cond = (coords or "").strip().lower(), (shape or "").strip()
    if system and system not in COORDS:
        raise ValueError(f"unknown coordinate system {system!r}; known: {', '.join(COORDS)}")
    if not cond:
        return pos, np.ones(pos.shape[:-1], bool)
    if not system:
        raise ValueError("a shape needs its coordinate system: set coords to one of " + ", ".join(COORDS))
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    if system == "cartesian":
        names = {"x": x, "y": y, "z": z}
    elif system == "spherical":
        r = np.sqrt(x * x + y * y + z * z)
        cos_t = np.divide(z, r, out=np.ones_like(z), where=r > 0)
        names = {"r": r, "theta": np.arccos(cos_t), "phi": np.arctan2(y, x)}
    else:
        names = {"rho": np.hypot(x, y), "phi": np.arctan2(y, x), "z": z}
    _validate_shape(cond, COORDS[system])
    keep = eval(compile(ast.parse(cond, mode="eval"), "<shape>", "eval"),   # every node checked above
                {"__builtins__": {}}, {**_FUNCS, **_CONSTS, **names})
    mask = np.broadcast_to(np.asarray(keep, bool), pos.shape[:-1]).copy()
    if not mask.any():
        raise ValueError(f"the shape {shape!r} contains no site of the box")
    return pos, mask


# -------------------------------------------------------------------------------------------- Hamiltonian
def _param(theta: dict, key: str, default: float = 0.0) -> float:
    v = theta.get(key, default)
    return float(default if v is None else v)


def dmi_matrices(crystal: cr.Crystal, D: float) -> dict[int, np.ndarray]:
    """Bulk-type (Bloch) DMI extra matrices A_lm = D sum_k r_k eps_klm on the in-plane first-shell bonds, r the
    unit bond vector (`simulate.py:153-168`)."""
    out = {}
    for i, bd in enumerate(crystal.bonds):
        if bd.shell != 1:
            continue
        r = np.zeros(3)
        d = np.asarray(bd.delta, float) + crystal.basis[bd.alpha2] - crystal.basis[bd.alpha]
        r[:crystal.D] = d @ crystal.vectors
        if abs(r[2]) > 1e-9:
            continue
        r /= np.linalg.norm(r)
        # sum_k r_k eps_klm is the cross-product matrix of r: (r x v)_l = sum_m A_lm v_m
        out[i] = D * np.array([[0.0, r[2], -r[1]], [-r[2], 0.0, r[0]], [r[1], -r[0], 0.0]])
    return out


def surface_sites(crystal: cr.Crystal, box, periodic, mask: np.ndarray) -> np.ndarray:
    """Active sites with fewer active first-shell neighbours than a bulk site of their basis index
    (`simulate.py:171-195`)."""
    bulk = np.zeros(crystal.b, int)
    count = np.zeros(mask.shape, int)
    sizes = [int(v) for v in box]
    for bd in crystal.bonds:
        if bd.shell != 1:
            continue
        bulk[bd.alpha] += 1
        nb = mask[bd.alpha2].astype(int)                 # (L3, L2, L1): is the neighbour across this bond active
        for k in range(crystal.D):
            d = bd.delta[k]
            if d == 0:
                continue
            ax = 2 - k                                   # lattice axis k -> array axis of (L3, L2, L1)
            nb = np.roll(nb, -d, axis=ax)
            if not periodic[k]:
                idx = np.arange(sizes[k])
                ok = ((idx + d) >= 0) & ((idx + d) < sizes[k])
                shp = [1, 1, 1]
                shp[ax] = sizes[k]
                nb = nb * ok.astype(int).reshape(shp)
        count[bd.alpha] += nb
    return mask & (count < bulk[:, None, None, None])


def build_system(model: str, crystal: str, box, periodic, theta: dict, mask=None, log=None) -> System:
    """The System of one state theta (J {shell: value}, D, K1, Ks, K2, H, H_theta, H_phi; `simulate.py:198-240`):
    exchange per shell, Bloch DMI and cubic anisotropy (Heisenberg only; K1 = Ks on surface sites), Zeeman
    field along (sin t cos p, sin t sin p, cos t) for Heisenberg, (cos p, sin p) for XY, +1 for Ising. A periodic
    box with no admissible colouring falls back to open boundaries."""
    name_m = str(model).strip().lower()
    if name_m not in MODELS:
        raise ValueError(f"unknown model {name_m!r}; known: {', '.join(MODELS)}")
    n = MODELS[name_m]
    J = {int(k): float(v) for k, v in (theta.get("J") or {1: 1.0}).items()}
    D, K1, K2, H = (_param(theta, k) for k in ("D", "K1", "K2", "H"))
    Ks = _param(theta, "Ks", K1)
    if n != 3 and any(_param(theta, k) for k in ("D", "K1", "Ks", "K2")):
        raise ValueError(f"D, K1, Ks and K2 need the Heisenberg model; {name_m} carries J and H only")
    unknown = set(theta) - {"name", "J", "D", "K1", "Ks", "K2", "H", "H_theta", "H_phi"}
    if unknown:
        raise ValueError(f"unknown parameters {sorted(unknown)}; known: J, D, K1, Ks, K2, H, H_theta, H_phi")
    shells = tuple(sorted({s for s, v in J.items() if v != 0.0} | {1}))
    c = cr.make(str(crystal), shells)
    box = tuple(int(v) for v in box)
    periodic = tuple(bool(v) for v in periodic)
    m = None if mask is None else np.asarray(mask, bool)
    want = (c.b, box[2] if c.D == 3 else 1, box[1], box[0])
    if m is not None and m.shape != want:
        raise ValueError(f"mask shape {m.shape} does not match the box {box} of {c.name}")
    h = None
    if H:
        t, p = np.deg2rad(_param(theta, "H_theta")), np.deg2rad(_param(theta, "H_phi"))
        direction = {1: (1.0,), 2: (np.cos(p), np.sin(p)),
                     3: (np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t))}[n]
        h = tuple(float(H * v) for v in direction)
    extra = dmi_matrices(c, D) if (n == 3 and D) else {}
    label = theta.get("name") or f"{name_m} {c.name}"

    def make(per):
        k1 = None
        if n == 3 and (K1 or Ks or K2):
            active = np.ones(want, bool) if m is None else m
            k1 = (np.where(surface_sites(c, box, per, active), Ks, K1) * active).astype(np.float32)
        return System(str(label), n, c, box, per, J, extra=extra, h=h, cubic_k1=k1, cubic_k2=K2, mask=m)

    try:
        return make(periodic)
    except ValueError as e:
        if not any(periodic) or "colouring" not in str(e):
            raise
        (log or print)(f"  no admissible colouring for the periodic box {box}: using open boundaries")
        return make((False,) * c.D)


# ---------------------------------------------------------------------------------------------------- a run
# The files of a run directory are the reference's (`simulate.py:20-26, 432-458, 492-494, 528-529`): run.json,
# sites.npy, mask.npy, configurations.npy (n_states, R, n_saved, n_sites, 3) float32, state_XXX_pYY.npz per state
# and replica block, magnetization.npy and results.npz from `collect` — same names, keys, dtypes and layout, so a
# directory written here loads with the reference's `load`.
def default_config() -> dict:
    """Every setting of a run with its default (a small sc Heisenberg ferromagnet)."""
    return dict(model="heisenberg", crystal="sc", box=[12, 12, 12], periodic=[True, True, True], coords="",
                shape="", states=[{"name": "J=1", "J": {"1": 1.0}}], units="reduced", T_max=2.0, T_min=0.2,
                T_step=0.1, thermalization=1000, measurement=2000, measure_every=10, replicas=32, config_every=1,
                seed=1)


def boltzmann(units: str) -> float:
    u = str(units).strip().lower()
    if u == "reduced":
        return 1.0
    if u == "mev":
        return KB_MEV
    raise ValueError("units must be 'reduced' (kB = 1) or 'meV' (T in kelvin)")


def size_estimate_gb(n_states: int, replicas: int, n_saved: int, n_sites: int) -> float:
    """Bytes of configurations.npy (float32, three components), in GB."""
    return n_states * replicas * n_saved * n_sites * 12 / 1e9


def replica_blocks(replicas: int, parts: int) -> list[tuple[int, int]]:
    """Replicas 0..R-1 in at most `parts` contiguous, non-empty blocks whose sizes differ by at most one."""
    R = int(replicas)
    k = max(1, min(int(parts), R))
    size, extra = divmod(R, k)
    bounds, start = [], 0
    for i in range(k):
        end = start + size + (1 if i < extra else 0)
        bounds.append((start, end))
        start = end
    return bounds


def prepare(cfg: dict, out, log=print) -> dict:
    """Validate a run, write run.json, sites.npy and mask.npy, and allocate configurations.npy."""
    out = Path(out)
    out.mkdir(parents=True, exist_ok=True)
    run_cfg = {**default_config(), **cfg}
    if not run_cfg["states"]:
        raise ValueError("define at least one state")
    kB = boltzmann(run_cfg["units"])
    temps = temperature_ladder(run_cfg["T_max"], run_cfg["T_min"], run_cfg["T_step"])
    pos, mask = active_sites(run_cfg["crystal"], run_cfg["box"], run_cfg["coords"], run_cfg["shape"])
    first = build_system(run_cfg["model"], run_cfg["crystal"], run_cfg["box"], run_cfg["periodic"],
                         run_cfg["states"][0], mask, log)
    every_t = max(1, int(run_cfg["config_every"]))
    n_saved = len(range(0, len(temps), every_t))
    n_sites = int(mask.sum())
    run_cfg.update(kB=kB, temperatures=temps.tolist(), periodic_used=list(first.periodic), n_sites=n_sites,
                   n_saved=n_saved, config_temperatures=temps[::every_t].tolist())
    for old in out.glob("state_*.npz"):          # blocks of an earlier run never mix with this one's
        old.unlink()
    (out / "run.json").write_text(json.dumps(run_cfg, indent=1))
    np.save(out / "sites.npy", pos[mask].astype(np.float32))
    np.save(out / "mask.npy", mask)
    shape = (len(run_cfg["states"]), int(run_cfg["replicas"]), n_saved, n_sites, 3)
    np.lib.format.open_memmap(out / "configurations.npy", mode="w+", dtype=np.float32, shape=shape).flush()
    log(f"{shape[0]} state(s) x {shape[1]} replicas x {len(temps)} temperatures, {n_sites} active sites; "
        f"configurations.npy = {size_estimate_gb(*shape[:4]):.3f} GB")
    return run_cfg


def run(cfg: dict, state_indices, out, device="cuda", log=print, replicas=None, part: int = 0,
        graphs: bool | None = None) -> None:
    """Simulate states of a prepared run for the replica block [r0, r1) (default: every replica) and write
    state_XXX_pYY.npz plus the block's slice of configurations.npy. Block `part` offsets the seed by 100000 per
    part (and each state by 1000), so blocks run on different GPUs are different chains."""
    out = Path(out)
    R = int(cfg["replicas"])
    r0, r1 = (0, R) if replicas is None else (int(replicas[0]), int(replicas[1]))
    if not 0 <= r0 < r1 <= R:
        raise ValueError(f"replica block [{r0}, {r1}) is outside 0..{R}")
    mask = np.load(out / "mask.npy")
    conf = np.load(out / "configurations.npy", mmap_mode="r+")
    for i in state_indices:
        theta = cfg["states"][i]
        log(f"state {i} ({theta.get('name', i)}), replicas {r0}-{r1 - 1}, on {device}")
        s = build_system(cfg["model"], cfg["crystal"], cfg["box"], cfg["periodic_used"], theta, mask, log)
        seed = int(cfg["seed"]) + 1000 * int(i) + 100000 * int(part)
        res = simulate_state(s, r1 - r0, cfg["temperatures"], int(cfg["thermalization"]), int(cfg["measurement"]),
                             int(cfg["measure_every"]), int(cfg["config_every"]), seed, device, float(cfg["kB"]),
                             log, graphs)
        conf[i, r0:r1] = res.pop("configs")
        conf.flush()
        np.savez(out / f"state_{i:03d}_p{int(part):02d}.npz", r0=r0, r1=r1, **res)
    del conf


def _blocks_of_state(out: Path, i: int, R: int) -> list:
    files = [np.load(f) for f in out.glob(f"state_{i:03d}_p*.npz")]
    files.sort(key=lambda z: int(z["r0"]))
    edge = 0
    for z in files:
        if int(z["r0"]) != edge:
            break
        edge = int(z["r1"])
    if not files or edge != R:
        raise ValueError(f"state {i}: its replica blocks do not cover replicas 0..{R - 1} exactly once")
    return files


def collect(out) -> dict:
    """Combine the state files of a run into arrays (n_states, replicas, nT[, 3]) plus Cv and chi per site
    (n_states, nT); writes magnetization.npy and results.npz."""
    out = Path(out)
    cfg = json.loads((out / "run.json").read_text())
    T = np.asarray(cfg["temperatures"])
    N, kB, R = float(cfg["n_sites"]), float(cfg["kB"]), int(cfg["replicas"])
    per_state = [_blocks_of_state(out, i, R) for i in range(len(cfg["states"]))]
    arr = {k: np.stack([np.concatenate([z[k] for z in files]) for files in per_state])
           for k in ("M", "E", "E2", "Mabs", "M2")}
    var_e = np.maximum(arr["E2"] - arr["E"] ** 2, 0.0)
    var_m = np.maximum(arr["M2"] - arr["Mabs"] ** 2, 0.0)
    res = dict(temperatures=T, magnetization=arr["M"], energy=arr["E"], energy2=arr["E2"], Mabs=arr["Mabs"],
               M2=arr["M2"], Cv=(var_e / (kB * T ** 2 * N)).mean(axis=1), chi=(N * var_m / (kB * T)).mean(axis=1),
               E_site=(arr["E"] / N).mean(axis=1), M_site=arr["Mabs"].mean(axis=1),
               state_names=np.array([str(st.get("name", i)) for i, st in enumerate(cfg["states"])]))
    np.save(out / "magnetization.npy", res["magnetization"])
    np.savez(out / "results.npz", **res)
    return res
