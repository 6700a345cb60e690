"""Replica split across processes / GPUs (one process per GPU, no exchange between chains).

Replicas are independent chains, so a multi-GPU run gives each rank a contiguous block of replicas and its own
seed offset (base + 100000 * rank), as the reference's `simulate.replica_blocks` / `api._run_on_gpus` do
(Spin_Colour_Kernel/simulate.py:461-468, api.py:126-150). The only inter-rank traffic is host-side bookkeeping:
the max of the timed regions and the gather of per-replica observables at the end.
"""

from __future__ import annotations

import torch

SEED_STRIDE = 100000


def replica_blocks(replicas: int, parts: int) -> list[tuple[int, int]]:
    """Split replicas 0..R-1 into at most `parts` contiguous blocks whose sizes differ by at most one."""
    R, g = int(replicas), max(1, min(int(parts), int(replicas)))
    q, r = divmod(R, g)
    edges = [0]
    for k in range(g):
        edges.append(edges[-1] + q + (1 if k < r else 0))
    return list(zip(edges[:-1], edges[1:]))


def rank_seed(base_seed: int, rank: int) -> int:
    return int(base_seed) + SEED_STRIDE * int(rank)


def max_over_ranks(value: float, group=None) -> float:
    """The largest of a float over all ranks (timings are the max over ranks)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_blocks(local: torch.Tensor, replicas: int, group=None) -> torch.Tensor:
    """Concatenate every rank's per-replica rows (rank order = replica order) into the full replica axis."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return local
    world = dist.get_world_size(group)
    blocks = replica_blocks(replicas, world)
    width = max(r1 - r0 for r0, r1 in blocks)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    out = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(out, pad, group=group)
    return torch.cat([o[: r1 - r0] for o, (r0, r1) in zip(out, blocks)])
