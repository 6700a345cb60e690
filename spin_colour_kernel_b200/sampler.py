"""Sampler: the reference's sampler interface over the B200 kernels of libsckb200.so.

Same constructor arguments, attributes, methods, device buffers and errors as
Spin_Colour_Kernel/sampler.py:39-345, so code written against the reference runs unchanged:
  Sampler(system, batch, device, seed, compact, spin_dtype, packed, bitwise, words_per_program, independent,
          bitwise_tile, bitwise_warps, max_block)
  .set_temperature(T)  .set_seed(seed, sweep)  .init_spins(kind, seed)  .pack(x)  .unpack(S)
  .sweep(S, n)  .graph(S, k)  .sync_sweep(S, n)  .reference_sweep(S, n)
  .local_field(S)  .energy(S)  .magnetization(S)
plus one keyword of its own, `layout`: "reference" (default) keeps S[B, n, b, L3, L2, L1]; "quad" keeps vector-model
spins interleaved four replicas per float4 with rows split by colour residue (include/sck.h, SCK_MODE_QUAD) —
the sampler's resident state, converted by pack / unpack as the reference converts its packed Ising words.
`state` (int64 {seed, sweep}), `beta` and the acceptance tables are device tensors updated in place, so a
captured CUDA graph keeps reading them by address. Every update runs in the CUDA kernels behind the C ABI of
include/sck.h; there is no CPU path, and a CPU device is refused.

The launch-geometry attributes of the reference (stride, bx, rows_per, block, chunks, cblock, cchunks, pblock,
pchunks, G, ngroups, ...) are computed with the reference's rules and kept for API compatibility; the CUDA
kernels choose their own tiling, and the chain does not depend on it.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from . import plan as P
from .system import System

COMPACT_MIN = 4
TILE = 128
MAX_BLOCK = 1024
PTILE = 64
WORD = 32
BWG = 4


def _num_warps(block: int) -> int:
    return 4 if block >= 256 else (2 if block >= 128 else 1)


def x_period(col) -> int:
    """Period along x of a linear colouring: lcm over its factors of m_r / gcd(K_r1, m_r)."""
    import math
    Pd = 1
    for r, mr in enumerate(col.m):
        Pd = math.lcm(Pd, mr // math.gcd(int(col.K[r][0]) % mr or mr, mr))
    return Pd


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


class Sampler:
    def __init__(self, system: System, batch: int, device="cuda", seed: int = 0, compact: bool = True,
                 spin_dtype: torch.dtype | None = None, packed: bool | None = None, bitwise: bool = False,
                 words_per_program: int | None = None, independent: bool = False, bitwise_tile: int | None = None,
                 bitwise_warps: int | None = None, max_block: int = MAX_BLOCK, layout: str = "reference"):
        self.sys = system
        if layout not in ("reference", "quad"):
            raise ValueError("layout must be 'reference' or 'quad'")
        self.layout = layout
        self.quad = layout == "quad"
        if self.quad and (system.n == 1 or bitwise or packed):
            raise ValueError("the interleaved 'quad' layout is for vector models (n = 2 or 3) in float32")
        self.bitwise = bool(bitwise)
        self.independent = bool(independent)
        if self.independent and not self.bitwise:
            raise ValueError("independent per-replica draws need bitwise=True")
        if self.bitwise:
            _, _, self.zmax = P.bitwise_check(system)
            if packed is False:
                raise ValueError("bitwise multi-spin coding uses the packed storage")
            packed = True
        self.packed = (system.n == 1 and int(batch) >= WORD) if packed is None else bool(packed)
        if self.packed and system.n != 1:
            raise ValueError("bit packing is for Ising (n = 1) only")
        self.spin_dtype = spin_dtype or (torch.int8 if system.n == 1 else torch.float32)
        if not self.packed and self.spin_dtype not in (torch.int8, torch.float32):
            raise ValueError("spin_dtype must be torch.int8 (Ising) or torch.float32")
        if self.spin_dtype == torch.int8 and system.n != 1:
            raise ValueError("int8 storage holds Ising spins only")
        self.B = int(batch)
        n, b, L3, L2, L1 = system.n, system.b, system.L3, system.L2, system.L1
        self.W = -(-self.B // WORD) if self.packed else self.B
        self.Bp = self.W * WORD if self.packed else (4 * -(-self.B // 4) if self.quad else self.B)
        self.Q = self.Bp // 4 if self.quad else 0
        if self.Bp * b * L3 * L2 * L1 >= 2 ** 31 - 1:
            raise ValueError("replica batch too large for the int32 Philox counter")
        gmax = words_per_program or BWG
        if gmax & (gmax - 1):
            raise ValueError("words_per_program must be a power of two")
        self.G = min(gmax, 1 << (self.W - 1).bit_length()) if self.bitwise else 1
        self.ngroups = -(-self.W // self.G)
        self.nrows = L3 * L2
        if max_block < 16 or max_block & (max_block - 1):
            raise ValueError("max_block must be a power of two >= 16")
        self._geometry(system, compact, bitwise_tile, bitwise_warps, max_block)
        if self.bitwise:
            self.mode = L.MODE_BITWISE_INDEP if self.independent else L.MODE_BITWISE
        elif self.packed:
            self.mode = L.MODE_PACKED
        elif self.quad:
            if self.spin_dtype != torch.float32:
                raise ValueError("the interleaved 'quad' layout stores float32 components")
            self.mode = L.MODE_QUAD
        elif self.spin_dtype == torch.int8:
            self.mode = L.MODE_INT8
        else:
            self.mode = L.MODE_F32
        self.desc = P.describe(system)
        lib = L.lib()
        handle = ctypes.c_void_p()
        L.check(lib.sck_plan_create(ctypes.byref(self.desc), self.B, self.mode, ctypes.byref(handle)))
        self._plan = handle
        nel, eb, keys = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
        L.check(lib.sck_plan_table_size(self._plan, ctypes.byref(nel), ctypes.byref(eb), ctypes.byref(keys)))
        self.keys = keys.value
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("spin_colour_kernel_b200 runs on CUDA devices (B200) only; there is no CPU path")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        dev = self.device
        m = system.site_mask()
        self.mask_np = m
        self.mask = torch.as_tensor(m.astype(np.int8), device=dev)
        k1 = system.cubic_k1 if system.cubic_k1 is not None else np.zeros(m.shape, np.float32)
        self.k1 = torch.as_tensor(np.asarray(k1, np.float32), device=dev)
        self.state = torch.tensor([int(seed), 0], dtype=torch.int64, device=dev)
        self.beta = torch.ones(self.Bp, dtype=torch.float32, device=dev)
        self.ptab = None
        self.lut = None
        if self.bitwise:
            self._table = P.p_fixed if self.independent else P.p_table
            self.ptab = torch.as_tensor(self._table(system, np.ones(self.W)), device=dev)
        elif system.n == 1:
            self.lut = torch.as_tensor(P.ising_table(system, np.ones(self.Bp, np.float32), self.keys), device=dev)
            assert self.lut.numel() == nel.value
        self.colours = system.colour_map()
        self.classes = P.sweep_classes(system)
        self._mask_f = torch.as_tensor(m, device=dev).to(torch.float32)
        self._obs_ws = {}
        self._flat_sampler = None
        self._workspace(self.B)

    def tune(self, specialised=True, l2_budget: int = 0, resident_limit: int = 200 << 10):
        """Execution choices of sweep: specialised kernels (1 or True: lattice kernels, the default; 2: segment
        kernels, 3: tile kernels, where the system allows them, else lattice kernels; 0 or False: generic),
        L2 group-pipeline budget
        (bytes), largest replica (bytes) whose sweeps run resident in shared memory. The chain does not depend on
        them."""
        level = int(specialised)
        L.check(L.lib().sck_plan_tune(self._plan, level, int(l2_budget), int(resident_limit)))
        return self.path()

    def pipeline(self, group: int, skew: int = 2, chunks: int | None = None):
        """Interleaved ('quad') layout only: run sweeps through the class-skewed L2 pipeline with groups of
        `group` replicas (a multiple of 4; 0 returns to class-by-class launches), class c of group-unit u at
        position skew * u + c, each ticket covering `chunks` site blocks (include/sck.h, sck_plan_pipeline,
        sck_plan_pipeline_chunks). The chain does not depend on it."""
        with torch.cuda.device(self.device):
            if chunks is not None:
                L.check(L.lib().sck_plan_pipeline_chunks(self._plan, int(chunks)))
            L.check(L.lib().sck_plan_pipeline(self._plan, int(group), int(skew)))
        return self.path()

    def set_wait_limit(self, polls: int):
        """Polls of a pipeline completion counter before a block gives up (failure-detection tests shorten it)."""
        L.check(L.lib().sck_plan_set_wait_limit(self._plan, int(polls)))

    def check_waits(self):
        """Synchronise the current stream and raise SckError (SCK_ERR_TIMEOUT) when a pipeline wait of this
        sampler gave up since the last check (its sites were left unchanged); clears the condition."""
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_plan_wait_status(self._plan, self._stream()))

    def path(self) -> dict:
        """The sweep path: specialised table id (0 = generic), budget, pipeline group, resident or not."""
        sp, bud, grp, res = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
        L.check(L.lib().sck_plan_path(self._plan, ctypes.byref(sp), ctypes.byref(bud), ctypes.byref(grp),
                                      ctypes.byref(res)))
        return {"specialised": sp.value, "l2_budget": bud.value, "group": grp.value, "resident": bool(res.value)}

    def __del__(self):
        h = getattr(self, "_plan", None)
        if h is not None and h.value:
            try:
                L.lib().sck_plan_destroy(h)
            except Exception:
                pass
            self._plan = None

    # ------------------------------------------------------------ reference launch geometry
    def _geometry(self, system, compact, bitwise_tile, bitwise_warps, max_block):
        L1 = system.L1
        self.block = min(max(16, 1 << (L1 - 1).bit_length()), max_block)
        self.chunks = -(-L1 // self.block)
        self.nw = _num_warps(self.block)
        Pd = x_period(system.colouring) if compact else 1
        Pd = Pd if Pd >= COMPACT_MIN else 1
        self.stride = Pd
        self.bx = -(-L1 // Pd)
        tile_c = bitwise_tile if (self.bitwise and bitwise_tile) else TILE
        self.rows_per = max(1, min(self.nrows, tile_c // self.bx)) if Pd > 1 else 1
        if self.packed and not self.bitwise:
            self.rows_per = max(1, min(self.nrows, PTILE // self.bx)) if Pd > 1 else 1
        self.cblock = max(16, 1 << (self.rows_per * self.bx - 1).bit_length())
        self.cchunks = 1
        if not self.packed and self.rows_per == 1 and self.cblock > max_block:
            self.cblock = max_block
            self.cchunks = -(-self.bx // max_block)
        self.cnw = _num_warps(self.cblock)
        if self.packed:
            nx = self.bx if Pd > 1 else L1
            tile = TILE if self.bitwise else PTILE
            self.pblock = min(tile, max(16, 1 << (nx - 1).bit_length()))
            self.pchunks = -(-nx // self.pblock)
            self.pblock_ref = min(tile, self.block)
            self.pchunks_ref = -(-L1 // self.pblock_ref)
            if not self.bitwise:
                self.cnw = 4 if self.cblock * WORD >= 2048 else 2
            elif bitwise_tile:
                self.pblock = min(bitwise_tile, max(16, 1 << (nx - 1).bit_length()))
                self.pchunks = -(-nx // self.pblock)
            if self.bitwise and bitwise_warps:
                self.cnw = self.nw = int(bitwise_warps)

    # ------------------------------------------------------------ state
    def set_temperature(self, T):
        T = torch.as_tensor(T, dtype=torch.float32).reshape(-1).cpu()
        beta = (1.0 / T).expand(self.B).contiguous() if T.numel() == 1 else (1.0 / T).contiguous()
        if beta.numel() != self.B:
            raise ValueError(f"need 1 or {self.B} temperatures, got {beta.numel()}")
        if self.Bp > self.B:     # padding replicas of the last word: computed, never observed
            beta = torch.cat([beta, beta[-1:].expand(self.Bp - self.B)])
        if self.bitwise:
            bwd = beta.reshape(self.W, WORD)
            if not torch.all(bwd == bwd[:, :1]):
                raise ValueError("bitwise multi-spin coding needs one temperature per word of 32 replicas")
            self.ptab.copy_(torch.as_tensor(self._table(self.sys, bwd[:, 0].double().numpy()), device=self.device))
        elif self.lut is not None:
            self.lut.copy_(torch.as_tensor(P.ising_table(self.sys, beta.numpy(), self.keys), device=self.device))
        self.beta.copy_(beta.to(self.device))

    def set_seed(self, seed: int, sweep: int = 0):
        self.state[0] = int(seed)
        self.state[1] = int(sweep)

    def init_spins(self, kind="random", seed: int = 0) -> torch.Tensor:
        s = self.sys
        g = torch.Generator(device="cpu").manual_seed(int(seed))
        shape = (self.B, s.n) + s.shape
        if kind == "ordered":
            x = torch.zeros(shape)
            x[:, 0] = 1.0
        elif s.n == 1:
            x = torch.randint(0, 2, shape, generator=g).float() * 2 - 1
        else:
            x = torch.randn(shape, generator=g)
            x = x / x.norm(dim=1, keepdim=True)
        x = x.to(self.device) * self._mask_f
        if self.packed or self.quad:
            return self.pack(x)
        return x.to(self.spin_dtype).contiguous()

    def quad_shape(self) -> tuple:
        """Shape of interleaved storage: (quads, b, L3, L2, n, L1, 4) float32."""
        s = self.sys
        return (self.Q, s.b, s.L3, s.L2, s.n, s.L1, 4)

    def _is_quad(self, S: torch.Tensor) -> bool:
        return self.quad and S.dim() == 7 and tuple(S.shape) == self.quad_shape()

    def pack(self, x: torch.Tensor) -> torch.Tensor:
        """(B, 1, b, L3, L2, L1) spins of +-1 (0 on masked sites) -> (W, 1, b, L3, L2, L1) int32 words; with the
        'quad' layout, (B, n, b, L3, L2, L1) float32 components -> interleaved quads (padding lanes 0)."""
        if self.quad:
            x = x.to(device=self.device, dtype=torch.float32).contiguous()
            if tuple(x.shape) != (self.B, self.sys.n) + self.sys.shape:
                raise ValueError(f"pack expects float32 spins of shape {(self.B, self.sys.n) + self.sys.shape}")
            out = torch.empty(self.quad_shape(), dtype=torch.float32, device=self.device)
            with torch.cuda.device(self.device):
                L.check(L.lib().sck_quad_pack(self._plan, _ptr(x), _ptr(out), self._stream()))
            return out
        sgn = (x > 0).to(torch.int8).to(self.device).contiguous()
        if sgn.shape[0] != self.B:
            raise ValueError("pack expects one row per replica")
        out = torch.empty((self.W, 1) + self.sys.shape, dtype=torch.int32, device=self.device)
        L.check(L.lib().sck_pack(self._plan, _ptr(sgn), _ptr(out), self._stream()))
        return out

    def unpack(self, S: torch.Tensor) -> torch.Tensor:
        """Packed words -> (B, 1, b, L3, L2, L1) int8 spins of +-1, 0 on masked sites; interleaved quads ->
        (B, n, b, L3, L2, L1) float32; identity for the reference layout."""
        if self._is_quad(S):
            self._check(S)
            out = torch.empty((self.B, self.sys.n) + self.sys.shape, dtype=torch.float32, device=self.device)
            with torch.cuda.device(self.device):
                L.check(L.lib().sck_quad_unpack(self._plan, _ptr(S), _ptr(out), self._stream()))
            return out
        if not self.packed or S.dtype != torch.int32:
            return S
        self._check(S)
        out = torch.empty((self.B, 1) + self.sys.shape, dtype=torch.int8, device=self.device)
        L.check(L.lib().sck_unpack(self._plan, _ptr(S), _ptr(self.mask), _ptr(out), self._stream()))
        return out

    # ------------------------------------------------------------ launches
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _check(self, S: torch.Tensor):
        want_dtype = torch.int32 if self.packed else self.spin_dtype
        want_shape = ((self.W, 1) if self.packed else (self.B, self.sys.n)) + self.sys.shape
        if self.quad:
            want_shape = self.quad_shape()
        if S.device != self.device or S.dtype != want_dtype or tuple(S.shape) != want_shape or not S.is_contiguous():
            raise ValueError(f"spins must be a contiguous {want_dtype} tensor of shape {want_shape} on {self.device}")

    def _buffers(self, S: torch.Tensor) -> L.Buffers:
        b = L.Buffers()
        b.spins = _ptr(S)
        b.mask = _ptr(self.mask) if self.sys.mask is not None else 0
        b.k1 = _ptr(self.k1) if self.sys.cubic_k1 is not None else 0
        b.beta = _ptr(self.beta)
        b.table = _ptr(self.ptab if self.bitwise else self.lut)
        b.state = _ptr(self.state)
        return b

    def sweep(self, S: torch.Tensor, n: int = 1) -> torch.Tensor:
        """n coloured sweeps in place; advances the sweep counter on the device."""
        self._check(S)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_sweep(self._plan, ctypes.byref(buf), int(n), self._stream()))
        return S

    def class_update(self, S: torch.Tensor, colour: int, alpha: int, src: torch.Tensor | None = None):
        """One class launch (the reference's kernel[grid](...) for class (colour, alpha))."""
        self._check(S)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_class_update(self._plan, ctypes.byref(buf), _ptr(src) if src is not None else None,
                                             int(colour), int(alpha), 0, self._stream()))
        return S

    def graph(self, S: torch.Tensor, k: int):
        """Capture k sweeps (launches and counter increments) in a CUDA graph; returns its replay."""
        with torch.cuda.device(self.device):
            return self._graph(S, k)

    def _graph(self, S: torch.Tensor, k: int):
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.sweep(S, 1)
        torch.cuda.current_stream(self.device).wait_stream(s)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.sweep(S, k)
        dev = self.device

        def replay():
            with torch.cuda.device(dev):
                g.replay()
        replay.keep = (self, S, g)
        return replay

    def _flat(self):
        """A reference-layout sampler over the same system, sharing this sampler's state and beta buffers (the
        checks that read S: synchronous control, sequential reference)."""
        if self._flat_sampler is None:
            f = Sampler(self.sys, self.B, device=self.device, seed=0)
            f.state = self.state
            f.beta = self.beta
            self._flat_sampler = f
        return self._flat_sampler

    def _via_flat(self, S, fn, n):
        X = self.unpack(S)
        getattr(self._flat(), fn)(X, n)
        S.copy_(self.pack(X))
        return S

    def sync_sweep(self, S: torch.Tensor, n: int = 1) -> torch.Tensor:
        """The negative control: every site updated in the same step from the old state."""
        if self.quad:
            return self._via_flat(S, "sync_sweep", n)
        self._check(S)
        scratch = torch.empty_like(S)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_sync_sweep(self._plan, ctypes.byref(buf), _ptr(scratch), int(n), self._stream()))
        return S

    def reference_sweep(self, S: torch.Tensor, n: int = 1) -> torch.Tensor:
        """Sequential reference chain on the GPU: classes in order, sites one at a time in raster order."""
        if self.quad:
            return self._via_flat(S, "reference_sweep", n)
        self._check(S)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_reference_sweep(self._plan, ctypes.byref(buf), int(n), self._stream()))
        return S

    # ------------------------------------------------------------ observables
    def local_field(self, S: torch.Tensor) -> torch.Tensor:
        """Bond part of the local field for every site (float64, torch rolls), a slow reference helper."""
        s = self.sys
        D = s.crystal.D
        S64 = self.unpack(S).double()
        v = torch.zeros_like(S64)
        dims = {0: 5, 1: 4, 2: 3}
        for i, bd in enumerate(s.crystal.bonds):
            M = torch.as_tensor(s.bond_matrix(i), dtype=torch.float64, device=S.device)
            if not M.any():
                continue
            src = S64[:, :, bd.alpha2]
            valid = torch.ones(s.shape[1:], dtype=torch.float64, device=S.device)
            for k in range(D):
                d = bd.delta[k]
                if d == 0:
                    continue
                src = torch.roll(src, shifts=-d, dims=dims[k] - 1)
                if not s.periodic[k]:
                    Lk = s.box[k]
                    idx = torch.arange(Lk, device=S.device)
                    ok = ((idx + d) >= 0) & ((idx + d) < Lk)
                    shp = [1, 1, 1]
                    shp[2 - k] = Lk
                    valid = valid * ok.to(torch.float64).reshape(shp)
            v[:, :, bd.alpha] += torch.einsum("kl,blzyx->bkzyx", M, src * valid)
        return v

    def _workspace(self, batch: int) -> torch.Tensor:
        ws = self._obs_ws.get(batch)
        if ws is None:
            nbytes = ctypes.c_int64()
            L.check(L.lib().sck_observables_workspace_size(self._plan, int(batch), ctypes.byref(nbytes)))
            ws = torch.empty(max(8, nbytes.value // 8), dtype=torch.float64, device=self.device)
            self._obs_ws[batch] = ws
        return ws

    def observables(self, S: torch.Tensor, E: torch.Tensor | None = None, M: torch.Tensor | None = None):
        """FP64 energy (B,) and per-sublattice magnetization (B, b, n) in one pass of the GPU reduction.

        S is this sampler's storage (packed words, int8 or float32 spins of any number of replicas).
        Graph-safe for the sampler's own batch: no host work, outputs may be preallocated."""
        s = self.sys
        if S.dtype == torch.int32 and self.packed:
            self._check(S)
            storage, batch = L.MODE_PACKED, self.B
        elif self._is_quad(S):
            self._check(S)
            storage, batch = L.MODE_QUAD, self.B
        else:
            if S.dtype == torch.int8 and s.n == 1:
                storage = L.MODE_INT8
            else:
                storage = L.MODE_F32
                if S.dtype != torch.float32:
                    S = S.to(torch.float32)
            S = S.contiguous()
            batch = int(S.shape[0])
            if tuple(S.shape[1:]) != (s.n,) + s.shape or S.device != self.device:
                raise ValueError(f"spins must have shape (batch, {s.n}) + {s.shape} on {self.device}")
        if E is None:
            E = torch.empty(batch, dtype=torch.float64, device=self.device)
        if M is None:
            M = torch.empty((batch, s.b, s.n), dtype=torch.float64, device=self.device)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_observables(self._plan, ctypes.byref(buf), _ptr(S), storage, batch, _ptr(E), _ptr(M),
                                            _ptr(self._workspace(batch)), self._stream()))
        return E, M

    def observe(self, S: torch.Tensor, E_ref: torch.Tensor, acc: torch.Tensor, accv: torch.Tensor,
                E: torch.Tensor, M: torch.Tensor):
        """One observation folded into FP64 accumulators on the device (the measure step of the ladder runner,
        simulate.py:338-353): with d = E - E_ref and m the mean magnetization vector, acc[0] += d,
        acc[1] += d^2, acc[2] += |m|, acc[3] += |m|^2 and accv += m, per replica. acc is (4, B), accv (B, n),
        E (B,) and M (B, b, n) receive the observation; all float64 on this device. Graph-safe."""
        s = self.sys
        B = self.B
        for t, shape in ((E_ref, (B,)), (E, (B,)), (M, (B, s.b, s.n)), (acc, (4, B)), (accv, (B, s.n))):
            if t.dtype != torch.float64 or tuple(t.shape) != shape or t.device != self.device or not t.is_contiguous():
                raise ValueError(f"observe wants contiguous float64 {shape} tensors on {self.device}")
        if S.dtype == torch.int32 and self.packed:
            self._check(S)
            storage = L.MODE_PACKED
        elif self._is_quad(S):
            self._check(S)
            storage = L.MODE_QUAD
        else:
            storage = L.MODE_INT8 if (S.dtype == torch.int8 and s.n == 1) else L.MODE_F32
            if storage == L.MODE_F32 and S.dtype != torch.float32:
                raise ValueError("observe reads this sampler's storage: int8, float32 or packed words")
            if tuple(S.shape) != (B, s.n) + s.shape or S.device != self.device or not S.is_contiguous():
                raise ValueError(f"spins must have shape ({B}, {s.n}) + {s.shape} on {self.device}")
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_observables_accumulate(
                self._plan, ctypes.byref(buf), _ptr(S), storage, B, float(s.n_active), _ptr(E_ref), _ptr(E),
                _ptr(M), _ptr(acc), _ptr(accv), _ptr(self._workspace(B)), self._stream()))

    def topological_charge(self, S: torch.Tensor, layer: int, Q: torch.Tensor | None = None) -> torch.Tensor:
        """Berg-Luscher charge (B,) float64 of z-layer `layer` of sublattice 0 (anneal.py:69-80). Graph-safe
        with a preallocated Q."""
        s = self.sys
        if self._is_quad(S):
            return self._flat().topological_charge(self.unpack(S), layer, Q)
        if S.dtype != torch.float32 or tuple(S.shape) != (self.B, s.n) + s.shape or not S.is_contiguous():
            raise ValueError(f"spins must be contiguous float32 ({self.B}, {s.n}) + {s.shape}")
        if Q is None:
            Q = torch.empty(self.B, dtype=torch.float64, device=self.device)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_topological_charge(self._plan, ctypes.byref(buf), _ptr(S), self.B, int(layer),
                                                   _ptr(Q), self._stream()))
        return Q

    def sweep_measure(self, S: torch.Tensor, n: int = 1, E: torch.Tensor | None = None,
                      M: torch.Tensor | None = None):
        """A measure step: n sweeps in place, then the FP64 energy (B,) and magnetization (B, b, n) of the state
        they leave (include/sck.h, sck_sweep_measure). With the 'quad' layout the last sweep accumulates them as it
        updates (float32 site shares, FP64 sums); otherwise it is sweep + observables. Graph-safe with
        preallocated outputs once the first call has sized the workspace."""
        self._check(S)
        s = self.sys
        if E is None:
            E = torch.empty(self.B, dtype=torch.float64, device=self.device)
        if M is None:
            M = torch.empty((self.B, s.b, s.n), dtype=torch.float64, device=self.device)
        ws = getattr(self, "_measure_ws", None)
        if ws is None:
            nbytes = ctypes.c_int64()
            L.check(L.lib().sck_sweep_measure_workspace_size(self._plan, ctypes.byref(nbytes)))
            ws = self._measure_ws = torch.empty(max(1, nbytes.value // 8), dtype=torch.float64, device=self.device)
        buf = self._buffers(S)
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_sweep_measure(self._plan, ctypes.byref(buf), int(n), _ptr(E), _ptr(M), _ptr(ws),
                                              self._stream()))
        return E, M

    def energy(self, S: torch.Tensor) -> torch.Tensor:
        """Total energy per replica, float64."""
        return self.observables(S)[0]

    def magnetization(self, S: torch.Tensor) -> torch.Tensor:
        """Per-sublattice magnetization M_alpha, shape (B, b, n), float64."""
        return self.observables(S)[1]


class SamplerBatch:
    """Several samplers (different systems, sizes, masks, colourings, temperatures) swept together.

    All samplers need the same storage (int8 Ising or float32 components of one spin dimension). A call is one
    persistent launch over per-system work descriptors: systems whose replica fits `resident_limit` bytes of
    shared memory run every sweep of the call on-chip, the rest class by class, each class waiting for the one
    before it in its own system (include/sck.h, sck_batch_*). Each sampler keeps its own spins, temperatures,
    tables and counter; `sweep(n)` advances every sampler's counter by n.
    """

    def __init__(self, samplers: list, spins: list, resident_limit: int = 200 << 10):
        if len(samplers) != len(spins) or not samplers:
            raise ValueError("one spins tensor per sampler")
        self.samplers = list(samplers)
        self.spins = list(spins)
        self.device = samplers[0].device
        arr = (ctypes.c_void_p * len(samplers))(*[s._plan.value for s in samplers])
        h = ctypes.c_void_p()
        L.check(L.lib().sck_batch_create(arr, len(samplers), int(resident_limit), ctypes.byref(h)))
        self._batch = h
        nbytes = ctypes.c_int64()
        L.check(L.lib().sck_batch_workspace_size(self._batch, ctypes.byref(nbytes)))
        self._ws = torch.empty(max(256, nbytes.value), dtype=torch.uint8, device=self.device)
        self.bind(spins)

    def bind(self, spins: list):
        """Point the batch at these spins tensors (and each sampler's current buffers); call outside capture."""
        for s, S in zip(self.samplers, spins):
            s._check(S)
        self.spins = list(spins)
        bufs = (L.Buffers * len(self.samplers))(*[s._buffers(S) for s, S in zip(self.samplers, spins)])
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_batch_bind(self._batch, bufs, _ptr(self._ws), self.samplers[0]._stream()))

    def info(self) -> dict:
        rs, rb, sb = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        L.check(L.lib().sck_batch_info(self._batch, ctypes.byref(rs), ctypes.byref(rb), ctypes.byref(sb)))
        return {"resident_systems": rs.value, "resident_blocks": rb.value, "step_blocks": sb.value}

    def sweep(self, n: int = 1):
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_batch_sweep(self._batch, _ptr(self._ws), int(n), self.samplers[0]._stream()))

    def set_wait_limit(self, polls: int):
        """Polls of a class wait before a block gives up (failure-detection tests shorten it)."""
        L.check(L.lib().sck_batch_set_wait_limit(self._batch, int(polls)))

    def check_waits(self):
        """Synchronise and raise SckError (SCK_ERR_TIMEOUT) when a wait of the batch kernel gave up since the last
        check (its sites were left unchanged); clears the condition."""
        with torch.cuda.device(self.device):
            L.check(L.lib().sck_batch_wait_status(self._batch, self.samplers[0]._stream()))

    def graph(self, k: int):
        """Capture k sweeps of the whole batch in a CUDA graph; returns its replay."""
        with torch.cuda.device(self.device):
            s = torch.cuda.Stream(device=self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                self.sweep(1)
            torch.cuda.current_stream(self.device).wait_stream(s)
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.sweep(k)
        dev = self.device

        def replay():
            with torch.cuda.device(dev):
                g.replay()
        replay.keep = (self, g)
        return replay

    def __del__(self):
        h = getattr(self, "_batch", None)
        if h is not None and h.value:
            try:
                L.lib().sck_batch_destroy(h)
            except Exception:
                pass
            self._batch = None
