"""Batched normals (se_normals_batch): many independent clouds of uneven sizes
and per-cloud k in one call, each cloud's result equal to a single-cloud call
on its own (bit-exact: same kNN, same normal arithmetic)."""
import numpy as np
import pytest

from shapeextraction_b200 import synth

pytestmark = pytest.mark.gpu


def _clouds(seed, n_clouds=23):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(50), np.log(60_000), n_clouds)).astype(int)
    sizes[3] = 0  # an empty cloud
    sizes[5] = 1
    sizes[7] = 17
    clouds = [synth.scene(int(s), seed=seed * 1000 + i) if s > 0 else
              (np.zeros(0, np.float32),) * 3 for i, s in enumerate(sizes)]
    ks = rng.choice([8, 16, 32], n_clouds).astype(np.int32)
    ks[9] = 5
    return clouds, ks


def test_batch_equals_single_cloud_calls(native):
    clouds, ks = _clouds(3)
    with native.Context() as c:
        nrm, offsets, u = c.normals_batch(clouds, ks)
        for i, (x, y, z) in enumerate(clouds):
            if x.size == 0:
                assert u[i] == 0
                continue
            c.build(x, y, z)
            assert u[i] == c.info()["n_points"]
            single = c.normals(int(ks[i]))
            assert np.array_equal(nrm[offsets[i]:offsets[i] + u[i]], single), i


def test_batch_repeated_and_device_resident(native):
    import torch

    clouds, ks = _clouds(4, 12)
    with native.Context() as c:
        a, offsets, u = c.normals_batch(clouds, ks)
        b, _, u2 = c.normals_batch(clouds, ks)
        assert np.array_equal(u, u2)
        for i in range(len(clouds)):
            assert np.array_equal(a[offsets[i]:offsets[i] + u[i]], b[offsets[i]:offsets[i] + u[i]])
        xs = [torch.from_numpy(np.concatenate([cl[j] for cl in clouds])).cuda() for j in range(3)]
        d, _, u3 = c.normals_batch(tuple(xs), (ks, offsets))
        d = d.cpu().numpy()
        assert np.array_equal(u, u3)
        for i in range(len(clouds)):
            assert np.array_equal(d[offsets[i]:offsets[i] + u[i]], a[offsets[i]:offsets[i] + u[i]])


def test_batch_rejects_bad_input(native):
    with native.Context() as c:
        x = np.zeros(10, np.float32)
        with pytest.raises(native.ShapexError):
            c.normals_batch([(x, x, x)], np.array([40], np.int32))  # k > 32
