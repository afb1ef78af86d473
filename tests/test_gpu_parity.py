"""GPU parity: every stage of the CUDA path, through the C ABI, against the
CPU oracle on the same seeded inputs.

Bar: bit-exact for codes, sort/dedup, radix tree, octree, decoded points and
kNN (indices and squared distances, ties by index); normals within 1e-3 rad
of the FP64 oracle where the neighbourhood is well conditioned."""
import numpy as np
import pytest

from shapeextraction_b200 import synth
from conftest import angle_deg_free

pytestmark = pytest.mark.gpu


def _ctx(native, **kw):
    return native.Context(**kw)


def _well_formed(oracle, x, y, z, bits):
    a = oracle.build_stages(x, y, z, bits, root_compat=True)["radix"]
    b = oracle.build_stages(x, y, z, bits, root_compat=False)["radix"]
    return all(np.array_equal(a[k][:1], b[k][:1]) for k in ("leftChild", "prefixN", "hasLeafLeft", "hasLeafRight"))


CLOUDS = [
    ("cube_30", lambda: synth.uniform_cube(20000, 11), 30),
    ("cube_63", lambda: synth.uniform_cube(20000, 12), 63),
    ("scene_63", lambda: synth.scene(50000, 13), 63),
    ("dups_63", lambda: synth.tiny_cloud(4000, 14), 63),
    ("mix_63", lambda: synth.precision_mix(40000, 15), 63),
]


@pytest.mark.parametrize("name,gen,bits", CLOUDS, ids=[c[0] for c in CLOUDS])
@pytest.mark.parametrize("compat", [True, False])
def test_build_stages_bit_exact(native, oracle, name, gen, bits, compat):
    x, y, z = gen()
    ref = oracle.build_stages(x, y, z, bits, root_compat=compat)
    with _ctx(native, code_bits=bits, root_compat=compat) as c:
        info = c.build(x, y, z)
        assert info["n_points"] == ref["codes"].size
        assert info["min_coord"] == ref["min"] and info["max_coord"] == ref["max"]
        assert np.array_equal(c.codes(), ref["codes"])
        assert np.array_equal(c.points(), ref["points"])
        r = c.radix()
        for key in ("leftChild", "prefixN", "hasLeafLeft", "hasLeafRight", "parent"):
            assert np.array_equal(r[key], ref["radix"][key]), key
        nodes = c.octree()
        assert info["n_octree"] == ref["octree"]["nodes"].size
        assert nodes.tobytes() == ref["octree"]["nodes"].tobytes()


def test_small_clouds_and_edge_sizes(native, oracle):
    """n = 1, 2, 3, all-duplicate clouds and small clouds around the compat-root quirk."""
    with _ctx(native) as c:
        for s in range(120):
            n = [1, 2, 3, 5, 8][s % 5] if s < 20 else 3 + s % 40
            x, y, z = synth.uniform_cube(n, seed=2000 + s)
            if s % 7 == 0:  # all duplicates
                x, y, z = np.full(n, 0.5, np.float32), np.full(n, 0.25, np.float32), np.full(n, 0.125, np.float32)
            ref = oracle.build_stages(x, y, z, 63, root_compat=True)
            info = c.build(x, y, z)
            u = ref["codes"].size
            assert info["n_points"] == u
            assert np.array_equal(c.codes(), ref["codes"])
            r = c.radix()
            for key in ("leftChild", "prefixN", "hasLeafLeft", "hasLeafRight"):
                assert np.array_equal(r[key], ref["radix"][key]), (s, key)
            if u >= 2 and _well_formed(oracle, x, y, z, 63):
                assert np.array_equal(r["parent"], ref["radix"]["parent"])
                assert c.octree().tobytes() == ref["octree"]["nodes"].tobytes()
            # the search always covers every point, whatever the compat root does
            k = 4
            idx, d2 = c.knn_self(k, with_d2=True)
            ei, ed = oracle.knn_exact(ref["points"], ref["points"], k)
            assert np.array_equal(idx, ei), s
            assert np.array_equal(d2, ed), s


def test_empty_cloud(native):
    with _ctx(native) as c:
        info = c.build(np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.float32))
        assert info["n_points"] == 0 and info["n_octree"] == 0
        assert c.normals(16).shape == (0, 3)


@pytest.mark.parametrize("k", [1, 5, 8, 10, 16, 20, 32])
@pytest.mark.parametrize("gen", ["cube", "scene"])
def test_knn_exact_bit_exact(native, oracle, k, gen):
    x, y, z = synth.uniform_cube(30000, 21) if gen == "cube" else synth.scene(60000, 22)
    with _ctx(native) as c:
        c.build(x, y, z)
        pts = c.points()
        idx, d2 = c.knn_self(k, with_d2=True)
        ei, ed = oracle.knn_exact(pts, pts, k)
        assert np.array_equal(d2, ed)
        assert np.array_equal(idx, ei)
        # a sub-range, as estimateNormals(octree, start, n) slices the queries
        s, n = 1234, 777
        i2 = c.knn_self(k, start=s, count=n)
        assert np.array_equal(i2, ei[s:s + n])


@pytest.mark.parametrize("bucket", [1, 4, 32, 33, 96, 128])
def test_knn_bucket_sizes(native, oracle, bucket):
    x, y, z = synth.scene(20000, 23)
    with _ctx(native, leaf_bucket=bucket) as c:
        c.build(x, y, z)
        pts = c.points()
        idx = c.knn_self(16)
        ei, _ = oracle.knn_exact(pts, pts, 16)
        assert np.array_equal(idx, ei)


def test_knn_lattice_ties(native, oracle):
    g = np.arange(24, dtype=np.float32) / 23.0
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    with _ctx(native) as c:
        c.build(gx.ravel().copy(), gy.ravel().copy(), gz.ravel().copy())
        pts = c.points()
        idx, d2 = c.knn_self(19, with_d2=True)
        ei, ed = oracle.knn_exact(pts, pts, 19)
        assert np.array_equal(idx, ei) and np.array_equal(d2, ed)


def test_knn_external_queries(native, oracle):
    x, y, z = synth.scene(40000, 24)
    rng = np.random.default_rng(5)
    q = rng.uniform(-0.2, 1.2, (5000, 3)).astype(np.float32)
    with _ctx(native) as c:
        c.build(x, y, z)
        pts = c.points()
        idx, d2 = c.knn(q, 16, with_d2=True)
        ei, ed = oracle.knn_exact(pts, q, 16)
        assert np.array_equal(d2, ed)
        assert np.array_equal(idx, ei)


@pytest.mark.parametrize("k", [8, 12, 16, 24, 32])
def test_normals_vs_fp64_oracle(native, oracle, k):
    x, y, z = synth.scene(60000, 31)
    with _ctx(native) as c:
        c.build(x, y, z)
        pts = c.points()
        nrm = c.normals(k)
        ei, _ = oracle.knn_exact(pts, pts, k)
        ref, ev = oracle.normals_f64(pts, ei, pts)
        gap = (ev[:, 1] - ev[:, 0]) / np.maximum(ev[:, 2], 1e-300)
        good = gap > 1e-4
        ang = angle_deg_free(nrm, ref)
        assert good.mean() > 0.95
        assert ang[good].max() <= 1e-3, ang[good].max()
        # sign convention: (viewpoint - p) . n >= 0 where it is not ambiguous
        dot = np.sum((0.0 - pts.astype(np.float64)) * nrm, axis=1)
        dref = np.sum((0.0 - pts.astype(np.float64)) * ref, axis=1)
        clear = good & (np.abs(dref) > 1e-4)
        assert np.all(dot[clear] >= 0)
        # unit length (no renormalisation, as the reference)
        assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-5)


def test_normals_near_degenerate_take_fp64(native, oracle):
    """Collinear points: tiny eigengap, so the FP64 path runs and still agrees
    with the FP64 oracle where the oracle's own normal is defined."""
    rng = np.random.default_rng(3)
    t = rng.random(20000)
    p = np.stack([t, 0.5 * t + 0.1, 0.25 * t + 0.2], 1) + rng.normal(0, 1e-6, (20000, 3))
    p = p.astype(np.float32)
    with _ctx(native, eigengap_fp64=1e-3) as c:
        c.build(p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy())
        pts = c.points()
        nrm = c.normals(16)
        assert c.stats()["fp64_solves"] > 0
        ei, _ = oracle.knn_exact(pts, pts, 16)
        ref, ev = oracle.normals_f64(pts, ei, pts)
        gap = (ev[:, 1] - ev[:, 0]) / np.maximum(ev[:, 2], 1e-300)
        ok = gap > 1e-3
        if ok.any():
            assert angle_deg_free(nrm[ok], ref[ok]).max() <= 1e-3


def test_normals_subrange_and_viewpoint(native, oracle):
    x, y, z = synth.scene(30000, 32)
    with _ctx(native, viewpoint=(5.0, -3.0, 2.0)) as c:
        c.build(x, y, z)
        pts = c.points()
        full = c.normals(16)
        part = c.normals(16, start=1000, count=4321)
        assert np.array_equal(part, full[1000:1000 + 4321])
        ei, _ = oracle.knn_exact(pts, pts, 16)
        ref, ev = oracle.normals_f64(pts, ei, pts, viewpoint=(5.0, -3.0, 2.0))
        d = np.sum((np.array([5.0, -3.0, 2.0]) - pts) * ref, axis=1)
        clear = np.abs(d) > 1e-3
        assert np.all(np.sum(full[clear] * ref[clear], axis=1) > 0)


def test_device_resident_inputs(native, oracle):
    import torch

    x, y, z = synth.scene(50000, 33)
    with _ctx(native) as c:
        c.build(x, y, z)
        host = c.normals(16)
        tx, ty, tz = (torch.from_numpy(a).cuda() for a in (x, y, z))
        c.build(tx, ty, tz)
        out = torch.zeros((c.info()["n_points"], 3), dtype=torch.float32, device="cuda")
        c.normals(16, out=out)
        assert np.array_equal(out.cpu().numpy(), host)


def test_errors_are_statuses(native):
    with _ctx(native) as c:
        with pytest.raises(native.ShapexError) as e:
            c.normals(16)
        assert e.value.status == 4  # not built
        x, y, z = synth.uniform_cube(1000, 1)
        x = x.copy()
        x[17] = np.nan
        with pytest.raises(native.ShapexError) as e:
            c.build(x, y, z)
        assert e.value.status == 5
        x[17] = np.inf
        with pytest.raises(native.ShapexError) as e:
            c.build(x, y, z)
        assert e.value.status == 5
        x[17] = 0.5
        c.build(x, y, z)
        with pytest.raises(native.ShapexError) as e:
            c.normals(33)
        assert e.value.status == 9
        with pytest.raises(native.ShapexError) as e:
            c.normals(16, start=10, count=10**7)
        assert e.value.status == 1
        # the context stays usable after errors
        assert c.normals(16).shape[0] == c.info()["n_points"]


def test_reference_api_facade(native, oracle):
    from shapeextraction_b200 import NormalEstimation, Octree, PointCloud, RadixTree

    x, y, z = synth.scene(20000, 34)
    cloud = PointCloud(x, y, z)
    rt = RadixTree(cloud)
    oc = Octree(rt)
    nrm = NormalEstimation.estimateNormals(oc, k=8)
    ref = oracle.build_stages(x, y, z)
    assert rt.n_pts == ref["codes"].size == oc.n_pts == nrm.shape[0]
    assert rt.n_nodes == rt.n_pts - 1
    assert oc.n_nodes == ref["octree"]["nodes"].size
    assert np.array_equal(oc.h_points, ref["points"])
    ei, _ = oracle.knn_exact(ref["points"], ref["points"][:100], 8)
    assert np.array_equal(oc.knnSearch(ref["points"][:100], 8), ei)


COMPAT_CLOUDS = [
    ("scene_200k_k16", lambda: synth.scene(200_000, 21), 16),
    ("cube_100k_k10", lambda: synth.uniform_cube(100_000, 22), 10),
    ("dups_20k_k8", lambda: synth.tiny_cloud(20_000, 23), 8),
    ("mix_60k_k32", lambda: synth.precision_mix(60_000, 24), 32),
]


@pytest.mark.parametrize("name,gen,k", COMPAT_CLOUDS, ids=[c[0] for c in COMPAT_CLOUDS])
def test_compat_search_bit_exact(native, oracle, name, gen, k):
    """Reference-compatible search mode: the reference's approximate neighbour
    lists (order included), self and external queries, against the oracle's
    restatement; normals against the restated reference pipeline."""
    x, y, z = gen()
    with _ctx(native, search_compat=True) as c:
        c.build(x, y, z)
        nodes = c.octree()
        pts = c.points()
        idx = c.knn_self(k)
        assert np.array_equal(idx, oracle.knn_compat(nodes, pts, pts, k))
        rng = np.random.default_rng(5)
        q = rng.uniform(-0.1, 1.1, (5000, 3)).astype(np.float32)
        q[:2500] = pts[rng.choice(pts.shape[0], 2500)] + rng.normal(0, 1e-3, (2500, 3)).astype(np.float32)
        assert np.array_equal(c.knn(q, k), oracle.knn_compat(nodes, pts, q, k))
        nrm = c.normals(k)
    u, ref = oracle.pipeline_reference(x, y, z, k)
    assert u == pts.shape[0]
    # both solve the same FP32 covariance in FP64; only (near-)repeated
    # eigenvalues leave the direction free
    _, ev = oracle.normals_f64(pts, idx, pts)
    gap = (ev[:, 1] - ev[:, 0]) / np.maximum(ev[:, 2], 1e-300)
    ok = gap > 1e-4
    assert ok.mean() > 0.5
    assert angle_deg_free(nrm[ok], ref[ok]).max() < 1e-4
    d = np.sum(-pts[ok].astype(np.float64) * ref[ok], axis=1)
    clear = np.abs(d) > 1e-4
    assert np.all(np.sum(nrm[ok][clear] * ref[ok][clear], axis=1) > 0)


def test_compat_search_rejections(native):
    x, y, z = synth.uniform_cube(1000, 3)
    with _ctx(native, search_compat=True, build_octree=False) as c:
        c.build(x, y, z)
        with pytest.raises(native.ShapexError):
            c.knn_self(8)
    with _ctx(native, search_compat=True) as c:
        with pytest.raises(native.ShapexError):
            c.normals_batch([(x, y, z)], np.array([8], np.int32))


def test_pinned_host_outputs_equal_device_outputs(native):
    """Pinned host outputs are written by the kernel directly (mapped host
    memory); pageable ones go through device staging. Both equal the
    device-output call bit for bit."""
    import torch

    x, y, z = synth.scene(300_000, 31)
    with _ctx(native) as c:
        u = c.build(x, y, z)["n_points"]
        n_dev = torch.empty((u, 3), dtype=torch.float32, device="cuda")
        c.normals(16, out=n_dev)
        n_pin = torch.zeros((u, 3), dtype=torch.float32).pin_memory()
        c.normals(16, out=n_pin)
        assert np.array_equal(n_pin.numpy(), n_dev.cpu().numpy())
        assert np.array_equal(c.normals(16), n_dev.cpu().numpy())  # pageable numpy output
        i_dev = torch.empty((u, 10), dtype=torch.int32, device="cuda")
        d_dev = torch.empty((u, 10), dtype=torch.float32, device="cuda")
        c.knn_self(10, out=i_dev, out_d2=d_dev)
        i_pin = torch.zeros((u, 10), dtype=torch.int32).pin_memory()
        d_pin = torch.zeros((u, 10), dtype=torch.float32).pin_memory()
        c.knn_self(10, out=i_pin, out_d2=d_pin)
        assert np.array_equal(i_pin.numpy(), i_dev.cpu().numpy()) and np.array_equal(d_pin.numpy(), d_dev.cpu().numpy())
        # a sub-range into the middle of a pinned buffer
        part = torch.zeros((u, 3), dtype=torch.float32).pin_memory()
        c.normals(16, 1000, 5000, out=part[1000:6000])
        assert np.array_equal(part[1000:6000].numpy(), n_dev[1000:6000].cpu().numpy())
        assert np.all(part[:1000].numpy() == 0) and np.all(part[6000:].numpy() == 0)
