"""Normal estimation sharded by query over ranks (one process per GPU).

Replaces the reference's MPI distribution (src/main.cu:17-47 bcastOctree,
src/main.cu:96-111 per-rank query counts and MPI_Gatherv) with
torch.distributed collectives (NCCL between GPUs, gloo on CPU):

1. The root rank's input coordinates are broadcast (12 bytes per point),
   instead of its octree (56 bytes per node plus the points): every rank
   builds the same tree itself. The build is deterministic, so all ranks agree
   on u, the Morton order and the tree; the ranks check that u matches.
2. The u Morton-ordered queries are split into contiguous ranges whose sizes
   differ by at most one. (The reference sizes every rank's receive count by
   its own rank's share, src/main.cu:104, which is wrong when u is not a
   multiple of the rank count.)
3. Each rank estimates the normals of its range; the ranges are gathered to
   every rank in rank order, which is Morton order.

There is no exchange inside the kNN step: ranks share nothing but the input
and the result, so the collectives are one broadcast and one all-gather.
"""
from __future__ import annotations

import numpy as np


def shard_ranges(u: int, world: int) -> list[tuple[int, int]]:
    """Contiguous (start, count) per rank covering [0, u); counts differ by at most one."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(max(int(u), 0), world)
    out, start = [], 0
    for r in range(world):
        c = base + (1 if r < extra else 0)
        out.append((start, c))
        start += c
    return out


def _device_for(group):
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _global_rank(group, group_rank: int) -> int:
    """The global rank of `group_rank` in `group` (collectives take global ranks)."""
    import torch.distributed as dist

    if group is None or group is dist.group.WORLD:
        return group_rank
    return dist.get_global_rank(group, group_rank)


def broadcast_cloud(x, y, z, group=None, root: int = 0):
    """The root's coordinates on every rank, as float32 tensors on the
    group's device (the other ranks may pass None). `root` is a rank within
    `group` (the default group: a global rank)."""
    import torch
    import torch.distributed as dist

    dev = _device_for(group)
    rank = dist.get_rank(group)
    src = _global_rank(group, root)
    n = torch.zeros(1, dtype=torch.int64, device=dev)
    if rank == root:
        n[0] = len(x)
    dist.broadcast(n, src=src, group=group)
    n = int(n[0])
    out = []
    for v in (x, y, z):
        if rank == root:
            t = torch.as_tensor(np.asarray(v, np.float32) if not torch.is_tensor(v) else v, dtype=torch.float32)
            t = t.to(dev).contiguous()
        else:
            t = torch.empty(n, dtype=torch.float32, device=dev)
        dist.broadcast(t, src=src, group=group)
        out.append(t)
    return tuple(out)


def sharded_normals(ctx, x, y, z, k: int, group=None, root: int = 0):
    """Normals of all u unique points (Morton order) on every rank, each rank
    computing one contiguous range. `ctx` is this rank's Context (or any
    object with build / info / normals of the same meaning); x, y, z are the
    root rank's coordinates (ignored elsewhere); `root` is a rank within
    `group`."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = _device_for(group)
    bx, by, bz = broadcast_cloud(x, y, z, group=group, root=root)
    if dev.type == "cpu":
        bx, by, bz = (t.numpy() for t in (bx, by, bz))
    u = int(ctx.build(bx, by, bz)["n_points"])
    # every rank must have built the same tree
    lo = torch.tensor([u], dtype=torch.int64, device=dev)
    hi = lo.clone()
    dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
    if int(lo[0]) != int(hi[0]):
        raise RuntimeError(f"ranks built different trees (u from {int(lo[0])} to {int(hi[0])})")
    ranges = shard_ranges(u, world)
    start, count = ranges[rank]
    width = max(c for _, c in ranges)  # equal-size pieces for the all-gather
    piece = torch.zeros((width, 3), dtype=torch.float32, device=dev)
    if count > 0:
        if dev.type == "cpu":
            piece[:count] = torch.from_numpy(np.asarray(ctx.normals(k, start, count), np.float32))
        else:
            ctx.normals(k, start, count, out=piece[:count])
    gathered = torch.empty((world * width, 3), dtype=torch.float32, device=dev)
    dist.all_gather_into_tensor(gathered, piece, group=group)
    parts = [gathered[r * width:r * width + c] for r, (_, c) in enumerate(ranges)]
    return torch.cat(parts, dim=0) if parts else gathered[:0]
