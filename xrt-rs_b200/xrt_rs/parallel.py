"""Several GPUs, one process each (torch.distributed).

Screen points are independent, so a solve shards by screen point with no
exchange during the compute: every rank solves a contiguous block of the
screen on its own GPU, and the blocks are gathered once at the end. With
device-resident blocks the gather is one all-gather of a (4, block) tensor
per rank over NCCL (NVLink), and the field never leaves the GPUs. The
benchmark's multi-GPU mode shards one solve this way (strong scaling) or runs
independent replicas (weak scaling); both time a step as the maximum over
ranks.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int):
    """[start, stop) of rank's block when n items are split as evenly as possible."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_screen(screen, rank: int, world: int):
    """This rank's block of screen points (dict of arrays) and its range."""
    n = len(screen["x"])
    a, b = shard_range(n, rank, world)
    return {k: np.ascontiguousarray(v[a:b]) for k, v in screen.items()}, (a, b)


def gather_field(local, n_total: int, group=None):
    """All-gather four float64 arrays of per-rank blocks into full arrays
    (blocks in rank order, lengths from shard_range)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = [shard_range(n_total, r, world) for r in range(world)]
    width = max(b - a for a, b in sizes)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    mine = torch.zeros(4, width, dtype=torch.float64, device=dev)
    a, b = sizes[rank]
    for c in range(4):
        mine[c, : b - a] = torch.as_tensor(np.asarray(local[c]), dtype=torch.float64)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = [np.empty(n_total, dtype=np.float64) for _ in range(4)]
    for r, (ra, rb) in enumerate(sizes):
        blk = parts[r].cpu().numpy()
        for c in range(4):
            out[c][ra:rb] = blk[c, : rb - ra]
    return tuple(out)


def gather_field_device(local, n_total: int, out=None, group=None):
    """All-gather this rank's block of the field, four 1-D tensors on its
    device (lengths from shard_range), into four full tensors on every rank
    (`out`, or new ones). One all-gather of a (4, width) tensor per rank: on
    NCCL the blocks move GPU to GPU; the gloo backend (CPU tensors) serves
    the host-side tests."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = [shard_range(n_total, r, world) for r in range(world)]
    width = max(b - a for a, b in sizes)
    dev = local[0].device
    a, b = sizes[rank]
    mine = torch.zeros(4, width, dtype=torch.float64, device=dev)
    for c in range(4):
        mine[c, : b - a].copy_(local[c])
    gathered = torch.empty(world, 4, width, dtype=torch.float64, device=dev)
    if dist.get_backend(group) == "nccl":
        dist.all_gather_into_tensor(gathered, mine, group=group)
    else:  # gloo has no single-tensor all-gather
        dist.all_gather(list(gathered.unbind(0)), mine, group=group)
    if out is None:
        out = [torch.empty(n_total, dtype=torch.float64, device=dev) for _ in range(4)]
    for r, (ra, rb) in enumerate(sizes):
        for c in range(4):
            out[c][ra:rb].copy_(gathered[r, c, : rb - ra])
    return out


def solve_sharded(rays, screen, compute=None, path="f32pr", ctx=None, group=None):
    """Solve one problem on every rank of `group`, each rank its block of the
    screen; returns the full field on every rank.

    `compute(rays, sub_screen) -> (es_re, es_im, ep_re, ep_im)` defaults to
    xrt_rs.diffraction_integral on this rank's current device.
    """
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sub, _ = shard_screen(screen, rank, world)
    if compute is None:
        import xrt_rs

        def compute(r, s):
            return xrt_rs.diffraction_integral(r, s, path=path, ctx=ctx)

    local = compute(rays, sub) if len(sub["x"]) else tuple(np.zeros(0) for _ in range(4))
    return gather_field(local, len(screen["x"]), group)


def max_over_ranks(value: float, group=None) -> float:
    """The maximum of a per-rank scalar (a step time) over the group."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
