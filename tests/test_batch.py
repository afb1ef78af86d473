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


def test_batch_graph_replay_equals_direct_launches(native):
    """The recorded graph (device or pinned host buffers) gives the same
    normals as plain launches, on first recording, on replay, after a layout
    change and when two layouts alternate."""
    import torch

    clouds, ks = _clouds(5, 17)
    clouds2, ks2 = _clouds(6, 11)
    with native.Context(batch_graph=False) as c:
        ref, offsets, u = c.normals_batch(clouds, ks)
        ref2, offsets2, u2 = c.normals_batch(clouds2, ks2)
    host = [torch.from_numpy(np.concatenate([cl[j] for cl in clouds])).pin_memory() for j in range(3)]
    host2 = [torch.from_numpy(np.concatenate([cl[j] for cl in clouds2])).pin_memory() for j in range(3)]
    dev = [h.cuda() for h in host]
    with native.Context(batch_graph=True) as c:
        out_h = torch.zeros((int(offsets[-1]), 3), dtype=torch.float32).pin_memory()
        out_h2 = torch.zeros((int(offsets2[-1]), 3), dtype=torch.float32).pin_memory()
        for rep in range(3):
            out_h.zero_()
            _, _, uu = c.normals_batch(tuple(host), (ks, offsets), out=out_h)
            assert np.array_equal(uu, u)
            assert np.array_equal(out_h.numpy(), ref), rep
            out_h2.zero_()
            _, _, uu2 = c.normals_batch(tuple(host2), (ks2, offsets2), out=out_h2)
            assert np.array_equal(uu2, u2)
            assert np.array_equal(out_h2.numpy(), ref2), rep
            d, _, uu = c.normals_batch(tuple(dev), (ks, offsets))
            assert np.array_equal(d.cpu().numpy(), ref), rep
        prof = c.profile()
        assert prof["query_launches"] == len(set(ks[u > 0].tolist())) + 1


@pytest.mark.parametrize("graph", [True, False])
def test_batch_large_and_small_clouds(native, graph):
    """Clouds large enough to be queried on their build lane next to small
    ones that share the persistent launch: every cloud equals its
    single-cloud call, through plain launches and through the graph."""
    import torch

    sizes = [150_000, 70_000, 3000, 500, 65_536, 65_535, 1, 0, 20_000]
    ks = np.array([16, 32, 8, 16, 10, 16, 8, 16, 5], np.int32)
    clouds = [synth.scene(s, seed=300 + i) if s > 0 else (np.zeros(0, np.float32),) * 3 for i, s in enumerate(sizes)]
    offsets = np.zeros(len(sizes) + 1, np.int64)
    offsets[1:] = np.cumsum(sizes)
    host = [torch.from_numpy(np.concatenate([cl[j] for cl in clouds])).pin_memory() for j in range(3)]
    with native.Context(batch_graph=graph) as c:
        out = torch.zeros((int(offsets[-1]), 3), dtype=torch.float32).pin_memory()
        for _ in range(2):
            out.zero_()
            _, _, u = c.normals_batch(tuple(host), (ks, offsets), out=out)
        nrm = out.numpy().copy()
        for i, (x, y, z) in enumerate(clouds):
            if x.size == 0:
                assert u[i] == 0
                continue
            c.build(x, y, z)
            assert u[i] == c.info()["n_points"]
            assert np.array_equal(nrm[offsets[i]:offsets[i] + u[i]], c.normals(int(ks[i]))), i


def test_batch_256_sampled_clouds_vs_oracle(native, oracle):
    """The batched configuration itself (256 scenes, sizes log-uniform in
    [1k, 500k], k per cloud from {8, 16, 32}; the bench's seed), checked
    against the CPU oracle rather than against single-cloud calls: for 8
    clouds of each k, spread over the sizes, the batch's u and normals (within
    1e-3 rad of FP64 where the FP64 relative eigengap exceeds 1e-4, with the
    reference's sign rule) and the cloud's self-query kNN lists (bit-exact)."""
    from conftest import angle_deg_free

    clouds, ks = synth.batched_clouds(256, 1)
    ks = np.ascontiguousarray(ks, np.int32)
    with native.Context() as c:
        nrm, offsets, u = c.normals_batch(clouds, ks)
        sizes = np.array([cl[0].size for cl in clouds])
        for k in (8, 16, 32):
            ids = np.flatnonzero(ks == k)
            ids = ids[np.argsort(sizes[ids])]
            pick = ids[np.linspace(0, ids.size - 1, min(8, ids.size)).astype(int)]
            for i in pick:
                x, y, z = clouds[i]
                ref = oracle.build_stages(x, y, z)
                pts = ref["points"]
                assert u[i] == pts.shape[0], i
                ei, ed = oracle.knn_exact(pts, pts, k)
                got = nrm[offsets[i]:offsets[i] + u[i]]
                nref, ev = oracle.normals_f64(pts, ei, pts)
                gap = (ev[:, 1] - ev[:, 0]) / np.maximum(np.abs(ev[:, 2]), 1e-300)
                good = gap > 1e-4
                assert good.mean() > 0.5, i
                assert angle_deg_free(got[good], nref[good]).max() <= 1e-3, i
                d = np.sum(-pts.astype(np.float64) * nref, axis=1)
                clear = good & (np.abs(d) > 1e-4)
                assert np.all(np.sum(got[clear] * nref[clear], axis=1) > 0), i
                c.build(x, y, z)
                idx, d2 = c.knn_self(k, with_d2=True)
                assert np.array_equal(d2, ed) and np.array_equal(idx, ei), i
