"""Learned block proposal for 3D Ising on the simple cubic lattice (include/sck_made.h).

No counterpart in the reference. A masked autoregressive MLP (MADE: 160 -> 256 -> 256 -> 256 -> 64, ReLU,
bfloat16 weights and activations, FP32 accumulation on tensor cores) proposes a joint update of a 4x4x4 block
conditioned on its 96 boundary spins; the proposal's exact density enters a Metropolis-Hastings ratio, so the
chain keeps the Boltzmann distribution whatever the network has learned. Blocks are coloured the way the sites of
a system are: `block_colouring` runs the colouring search on the graph of blocks (two blocks interact when they
touch at a face, an edge or a corner), verifies it bond by bond on the periodic block box and certifies it against
the clique number; blocks of one colour share no bond and neither touches another's boundary, so a colour step
updates them all at once. `round` runs one colour step per colour in the colouring's order, after which the caller
interleaves plain colour sweeps (`Sampler.sweep`) on the same int8 spins.

`BlockProposal.train` fits the network on block inputs gathered from configurations of the plain chain
(`gather`), with the library's own forward and backward kernels and Adam. Everything runs on the GPU through
libsckb200.so; there is no CPU path.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as abi

IN, HIDDEN, SPINS, BOUNDARY = 160, 256, 64, 96
NPARAM = 256 * 160 + 256 + 2 * (256 * 256 + 256) + 64 * 256 + 64
SHAPES = [((256, 160), (256,)), ((256, 256), (256,)), ((256, 256), (256,)), ((64, 256), (64,))]


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def block_colouring(nb: int):
    """(colouring, parity code per colour) of the nb^3 periodic lattice of 4x4x4 blocks.

    The block graph is the simple cubic lattice of blocks with its first three shells (face, edge and corner
    neighbours), and its colouring is found by the same search as a system's site colouring
    (`colouring.search`, first admissible linear colouring by increasing colour count), then checked bond by bond
    on the box and against the clique number (the 2x2x2 cube of blocks is a clique of 8). The colour-step kernel
    addresses the blocks of a class by the parities of their block coordinates, code px + 2 py + 4 pz; every
    class must therefore be one parity coset, which is checked here."""
    from . import colouring as co
    from . import crystals as cr
    if nb < 2 or nb % 2:
        raise ValueError("the block lattice needs an even number of blocks per axis")
    crystal = cr.make("sc", (1, 2, 3))
    box, per = (nb, nb, nb), (True, True, True)
    col = co.search(crystal, box, per)
    if col is None or not co.verify_on_box(col, crystal, box, per):
        raise ValueError("no verified block colouring of the block lattice")
    if col.n_colours != co.clique_number(crystal):
        raise ValueError(f"block colouring of {col.n_colours} colours is not optimal")
    grid = col.colour_grid(0, box)                      # (z, y, x)
    z, y, x = np.meshgrid(np.arange(nb), np.arange(nb), np.arange(nb), indexing="ij")
    parity = (x % 2) + 2 * (y % 2) + 4 * (z % 2)
    codes = []
    for c in range(col.n_colours):
        p = np.unique(parity[grid == c])
        if p.size != 1 or np.any(grid[parity == p[0]] != c):
            raise ValueError("a block colour class is not a parity class of the block coordinates")
        codes.append(int(p[0]))
    return col, codes


def kaiming_params(seed: int = 0):
    """[(W, b)] float32: uniform(+-sqrt(6 / fan_in)) weights, zero biases (NumPy PCG64 from `seed`)."""
    rng = np.random.default_rng(seed)
    out = []
    for (wshape, bshape) in SHAPES:
        bound = np.sqrt(6.0 / wshape[1])
        out.append((rng.uniform(-bound, bound, wshape).astype(np.float32), np.zeros(bshape, np.float32)))
    return out


def flatten(params) -> np.ndarray:
    return np.concatenate([np.concatenate([W.reshape(-1), b.reshape(-1)]) for W, b in params]).astype(np.float32)


def unflatten(flat: np.ndarray):
    out, o = [], 0
    for (wshape, bshape) in SHAPES:
        nw, nb = wshape[0] * wshape[1], bshape[0]
        out.append((flat[o:o + nw].reshape(wshape).copy(), flat[o + nw:o + nw + nb].copy()))
        o += nw + nb
    return out


class BlockProposal:
    """Network parameters, Adam moments and the colour steps of the learned block proposal on one GPU.

    L: lattice edge (multiple of 8); R: replicas; groups: autoregressive steps per block (16: four mutually
    non-adjacent spins per step; 64: one spin per step)."""

    def __init__(self, L: int, R: int, groups: int = 16, seed: int = 0, device="cuda", params=None):
        if L % 8 or L < 8:
            raise ValueError("L must be a multiple of 8")
        if groups not in (16, 64):
            raise ValueError("groups must be 16 or 64")
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("the learned proposal runs on a CUDA device only")
        self.device = torch.device("cuda", dev.index if dev.index is not None else torch.cuda.current_device())
        self.L, self.R, self.groups = int(L), int(R), int(groups)
        self.nb = self.L // 4
        self.block_colouring, self.colour_codes = block_colouring(self.nb)
        pb, ab = ctypes.c_int64(), ctypes.c_int64()
        abi.check(abi.lib().sck_made_sizes(self.groups, 64, ctypes.byref(pb), ctypes.byref(ab), None))
        self.params = torch.zeros(pb.value, dtype=torch.uint8, device=self.device)
        self.adam = torch.zeros(ab.value // 4, dtype=torch.float32, device=self.device)
        self.t = 0
        self._ws = {}
        self.set_params(params if params is not None else kaiming_params(seed))

    # ------------------------------------------------------------------ parameters
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def masters(self) -> torch.Tensor:
        """FP32 master parameters (a view into the parameter buffer)."""
        return self.params[: NPARAM * 4].view(torch.float32)

    def set_params(self, params) -> None:
        flat = torch.from_numpy(flatten(params)).to(self.device)
        self.masters().copy_(flat)
        self.adam.zero_()
        self.t = 0
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_prepare(_ptr(self.params), self.groups, self._stream()))

    def get_params(self):
        return unflatten(self.masters().cpu().numpy())

    def _workspace(self, batch: int) -> torch.Tensor:
        if batch not in self._ws:
            tb = ctypes.c_int64()
            abi.check(abi.lib().sck_made_sizes(self.groups, batch, None, None, ctypes.byref(tb)))
            self._ws[batch] = torch.empty(tb.value, dtype=torch.uint8, device=self.device)
        return self._ws[batch]

    # ------------------------------------------------------------------ data and training
    def gather(self, spins: torch.Tensor) -> torch.Tensor:
        """Block inputs (bfloat16, [R nb^3, 160]) of every block of int8 spins [R, 1, 1, L, L, L] or [R, L, L, L]."""
        S = spins.contiguous()
        R = S.shape[0]
        if S.dtype != torch.int8 or S.numel() != R * self.L ** 3 or S.device != self.device:
            raise ValueError(f"spins must be int8 with {self.L}^3 sites per replica on {self.device}")
        out = torch.empty((R * self.nb ** 3, IN), dtype=torch.bfloat16, device=self.device)
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_gather(_ptr(S), R, self.L, _ptr(out), self._stream()))
        return out

    def forward(self, x: torch.Tensor):
        """(logits [n, 64] FP32, log q [n] FP32) of block-input rows x (bfloat16, n a multiple of 64)."""
        n = x.shape[0]
        logits = torch.empty((n, SPINS), dtype=torch.float32, device=self.device)
        logq = torch.empty(n, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_forward(_ptr(self.params), self.groups, _ptr(x.contiguous()), n,
                                                 _ptr(logits), _ptr(logq), _ptr(self._workspace(n)), self._stream()))
        self.check_waits()
        return logits, logq

    def check_waits(self) -> None:
        """Synchronise the current stream and raise SckError (SCK_ERR_TIMEOUT) when a bounded wait of the
        tensor-core GEMM gave up on this device since the last check (its output rows were left unwritten)."""
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_wait_status(self._stream()))

    def set_wait_limit(self, polls: int) -> None:
        """Polls of a GEMM stage's mbarrier before a block gives up, on this device (failure-detection tests
        shorten it; the default is 2^22)."""
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_set_wait_limit(int(polls)))

    def grads(self, x: torch.Tensor):
        """(loss, [(dW, db)] as float32 NumPy) of the mean negative log-density of rows x."""
        n = x.shape[0]
        g = torch.empty(NPARAM, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_grads(_ptr(self.params), self.groups, _ptr(x.contiguous()), n, _ptr(g),
                                               _ptr(loss), _ptr(self._workspace(n)), self._stream()))
        return float(loss.item()), unflatten(g.cpu().numpy())

    def train(self, data: torch.Tensor, steps: int, batch: int = 8192, lr: float = 1e-3, betas=(0.9, 0.999),
              eps: float = 1e-8, seed: int = 0):
        """Adam on minibatches drawn (without replacement within an epoch) from `data` rows; returns the loss of
        every step (one device-to-host read at the end)."""
        n = data.shape[0]
        if batch % 64 or batch > n:
            raise ValueError("batch must be a multiple of 64 and at most the number of rows")
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        losses = torch.empty(steps, dtype=torch.float32, device=self.device)
        ws = self._workspace(batch)
        perm = torch.randperm(n, device=self.device, generator=gen)
        pos = 0
        xb = torch.empty((batch, IN), dtype=torch.bfloat16, device=self.device)
        with torch.cuda.device(self.device):
            for i in range(steps):
                if pos + batch > n:
                    perm = torch.randperm(n, device=self.device, generator=gen)
                    pos = 0
                torch.index_select(data, 0, perm[pos:pos + batch], out=xb)
                pos += batch
                self.t += 1
                abi.check(abi.lib().sck_made_train_step(_ptr(self.params), _ptr(self.adam), self.groups, _ptr(xb),
                                                        batch, lr, betas[0], betas[1], eps, self.t,
                                                        _ptr(losses[i:i + 1]), _ptr(ws), self._stream()))
        self.check_waits()
        return losses.cpu().numpy()

    # ------------------------------------------------------------------ sampling
    def colour_step(self, spins: torch.Tensor, beta: torch.Tensor, colour: int, seed: int, rnd: int,
                    accepted: torch.Tensor | None = None, record: torch.Tensor | None = None) -> None:
        """One colour step in place on int8 spins of this proposal's R replicas (beta: FP32 per replica); `colour`
        is the class's parity code (px + 2 py + 4 pz of its blocks' coordinates)."""
        with torch.cuda.device(self.device):
            abi.check(abi.lib().sck_made_colour_step(_ptr(self.params), self.groups, _ptr(spins), self.R, self.L,
                                                     _ptr(beta), int(colour), int(seed), int(rnd), _ptr(accepted),
                                                     _ptr(record), self._stream()))

    def round(self, spins: torch.Tensor, beta: torch.Tensor, seed: int, rnd: int,
              accepted: torch.Tensor | None = None) -> None:
        """The colour steps of block round `rnd`, one per colour of the block colouring, in its order."""
        for code in self.colour_codes:
            self.colour_step(spins, beta, code, seed, rnd, accepted)

    def record_buffer(self) -> torch.Tensor:
        """A record buffer for colour_step: 80 bytes per (replica, block of the colour)."""
        return torch.zeros(self.R * (self.nb ** 3 // 8) * 80, dtype=torch.uint8, device=self.device)

    @staticmethod
    def parse_record(rec: torch.Tensor, R: int, nc: int):
        """(x' int8 [R, nc, 64], log q(x') [R, nc], log q(x) [R, nc], dE [R, nc], accepted [R, nc])."""
        a = rec.view(R * nc, 80).cpu()
        xs = a[:, :64].view(torch.int8).reshape(R, nc, 64).numpy()
        f = a[:, 64:].contiguous().view(torch.float32).reshape(R, nc, 4).numpy()
        return xs, f[..., 0], f[..., 1], f[..., 2], f[..., 3] > 0.5
