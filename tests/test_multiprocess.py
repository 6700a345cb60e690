"""The multi-rank path on the CPU: world_size 2 over gloo. Each rank runs its replica block with its own seed
offset (the oracle stands in for the GPU chain), the ranks agree on the max of their timings, and the gathered
per-replica observables cover every replica exactly once with distinct chains."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from spin_colour_kernel_b200 import replicas as RP


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, R, out):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import observables as obs
        from oracle import sweep as osw
        from spin_colour_kernel_b200 import system as sy
        s = sy.ising("square", 8)
        r0, r1 = RP.replica_blocks(R, world)[rank]
        g = torch.Generator().manual_seed(RP.rank_seed(7, rank))
        S = (torch.randint(0, 2, (r1 - r0, 1) + s.shape, generator=g) * 2 - 1).to(torch.int8).numpy()
        beta = np.full(r1 - r0, np.float32(1.0) / np.float32(2.3), np.float32)
        osw.sweep(s, S, beta, [RP.rank_seed(1234, rank), 0], 3)
        E = torch.from_numpy(obs.energy(s, S))
        slowest = RP.max_over_ranks(0.5 + rank)
        allE = RP.gather_blocks(E, R)
        allS = RP.gather_blocks(torch.from_numpy(S.reshape(r1 - r0, -1).astype(np.int64)), R)
        if rank == 0:
            out.put((slowest, allE.numpy(), allS.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_replicas_and_gather():
    assert RP.replica_blocks(10, 4) == [(0, 3), (3, 6), (6, 8), (8, 10)]
    assert RP.replica_blocks(32, 2) == [(0, 16), (16, 32)]
    assert RP.replica_blocks(3, 8) == [(0, 1), (1, 2), (2, 3)]
    R, world = 5, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, R, q)) for r in range(world)]
    for p in procs:
        p.start()
    slowest, E, S = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert slowest == 1.5
    assert E.shape == (R,) and S.shape[0] == R
    assert np.all(np.abs(S) == 1)                         # every replica slot came from a chain
    assert not np.array_equal(S[0], S[3])                 # different ranks run different chains
