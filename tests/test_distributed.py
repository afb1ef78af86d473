"""Query sharding (shapeextraction_b200/distributed.py): the host logic runs
as two gloo ranks on CPU with a stand-in for the GPU context; the NCCL path
runs on one GPU through the real context."""
import os
import socket

import numpy as np
import pytest

from shapeextraction_b200.distributed import shard_ranges


def test_shard_ranges_cover_and_balance():
    for u in (0, 1, 2, 3, 7, 100, 1_000_003):
        for world in (1, 2, 3, 8):
            r = shard_ranges(u, world)
            assert len(r) == world
            assert sum(c for _, c in r) == u
            assert all(r[i][0] + r[i][1] == r[i + 1][0] for i in range(world - 1))
            counts = [c for _, c in r]
            assert max(counts) - min(counts) <= 1


class _StubContext:
    """Stands in for a Context on CPU: 'builds' by sorting unique points and
    returns a normal that encodes the global query index."""

    def build(self, x, y, z):
        pts = np.unique(np.stack([x, y, z], 1), axis=0)
        self.u = pts.shape[0]
        return {"n_points": self.u}

    def normals(self, k, start, count):
        i = np.arange(start, start + count, dtype=np.float32)
        return np.stack([i, 2 * i + k, -i], 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, results):
    import torch.distributed as dist

    from shapeextraction_b200.distributed import sharded_normals

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(0)
        x, y, z = (rng.integers(0, 50, n).astype(np.float32) for _ in range(3)) if rank == 0 else (None,) * 3
        out = sharded_normals(_StubContext(), x, y, z, 8)
        results[rank] = out.numpy()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [0, 1, 3, 1001])
def test_sharded_normals_two_gloo_ranks(n):
    import torch.multiprocessing as mp

    world = 2
    mgr = mp.Manager()
    results = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), n, results), nprocs=world, join=True)
    rng = np.random.default_rng(0)
    x, y, z = (rng.integers(0, 50, n).astype(np.float32) for _ in range(3))
    u = _StubContext().build(x, y, z)["n_points"]
    want = _StubContext().normals(8, 0, u)
    for r in range(world):
        assert results[r].shape == (u, 3)
        assert np.array_equal(results[r], want)


def _subgroup_worker(rank, world, port, n, results):
    import torch.distributed as dist

    from shapeextraction_b200.distributed import sharded_normals

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # a subgroup of global ranks {1, 2}; its rank 0 (global rank 1) is the root
        sub = dist.new_group([1, 2])
        if rank in (1, 2):
            rng = np.random.default_rng(0)
            x, y, z = (rng.integers(0, 50, n).astype(np.float32) for _ in range(3)) if rank == 1 else (None,) * 3
            out = sharded_normals(_StubContext(), x, y, z, 8, group=sub, root=0)
            results[rank] = out.numpy()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_normals_subgroup_root_is_a_group_rank():
    """`root` names a rank of the group, not a global rank: in a subgroup of
    global ranks {1, 2}, root 0 is global rank 1, the only rank holding data."""
    import torch.multiprocessing as mp

    n = 777
    mgr = mp.Manager()
    results = mgr.dict()
    mp.spawn(_subgroup_worker, args=(3, _free_port(), n, results), nprocs=3, join=True)
    rng = np.random.default_rng(0)
    x, y, z = (rng.integers(0, 50, n).astype(np.float32) for _ in range(3))
    u = _StubContext().build(x, y, z)["n_points"]
    want = _StubContext().normals(8, 0, u)
    assert sorted(results.keys()) == [1, 2]
    for r in (1, 2):
        assert np.array_equal(results[r], want)


@pytest.mark.gpu
def test_sharded_normals_one_nccl_rank(native):
    import torch
    import torch.distributed as dist

    from shapeextraction_b200 import synth
    from shapeextraction_b200.distributed import sharded_normals

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        x, y, z = synth.scene(50_000, 9)
        with native.Context() as c:
            got = sharded_normals(c, x, y, z, 16).cpu().numpy()
            c.build(x, y, z)
            assert np.array_equal(got, c.normals(16))
    finally:
        dist.destroy_process_group()
