"""CPU checks of the oracle itself: each restated stage against an independent
slow restatement or invariant. The oracle is pinned against the reference's
own outputs in test_golden.py."""
import numpy as np
import pytest

from shapeextraction_b200 import synth


def slow_encode(x, y, z, mn, rng, bits):
    """Bit-by-bit pointToCode (src/MortonUtils.cu:7-19) in numpy float32."""
    bpa = bits // 3
    bs = np.float32((1 << bpa) - 1)
    out = []
    for a, b, c in zip(x, y, z):
        q = []
        for v in (a, b, c):
            f = np.float32(bs * np.float32(np.float32(v - np.float32(mn)) / np.float32(rng)))
            q.append(int(f) & ((1 << bpa) - 1))
        code = 0
        for i in range(bpa):
            for ax in range(3):
                code |= ((q[ax] >> i) & 1) << (3 * i + ax)
        out.append(code)
    return np.array(out, np.uint64)


@pytest.mark.parametrize("bits", [30, 63])
def test_encode_matches_bitwise(oracle, bits):
    x, y, z = synth.uniform_cube(500, seed=3)
    mn, mx = oracle.bbox(x, y, z)
    got = oracle.encode(x, y, z, mn, mx - mn, bits)
    assert np.array_equal(got, slow_encode(x, y, z, mn, mx - mn, bits))


def test_bbox_is_isotropic_min_max(oracle):
    x, y, z = synth.scene(5000, seed=2)
    mn, mx = oracle.bbox(x, y, z)
    assert mn == min(x.min(), y.min(), z.min())
    assert mx == max(x.max(), y.max(), z.max())


def test_decode_fma_and_roundtrip(oracle):
    rng = np.random.default_rng(0)
    q = rng.integers(0, 1 << 21, (1000, 3)).astype(np.uint64)
    codes = np.zeros(1000, np.uint64)
    for i in range(21):
        for ax in range(3):
            codes |= ((q[:, ax] >> np.uint64(i)) & np.uint64(1)) << np.uint64(3 * i + ax)
    mn, rg = np.float32(-0.37), np.float32(2.5)
    pts = oracle.decode(codes, float(mn), float(rg), 63)
    # codeToPoint: fmaf(raw / bitscale, range, min)
    f = (q.astype(np.float32) / np.float32(2097151.0)).astype(np.float32)
    ref = (f.astype(np.float64) * np.float64(rg) + np.float64(mn)).astype(np.float32)  # single rounding == fma
    assert np.array_equal(pts, ref)


def test_sort_dedup(oracle):
    x, y, z = synth.tiny_cloud(3000, seed=4)
    mn, mx = oracle.bbox(x, y, z)
    c = oracle.encode(x, y, z, mn, mx - mn)
    assert np.array_equal(oracle.sort_dedup(c), np.unique(c))


def _subtree_leaves(radix, u, root_gamma, root_hl, root_hr):
    """Leaves reachable from the root, walking children (full tree)."""
    lc, hl, hr = radix["leftChild"], radix["hasLeafLeft"], radix["hasLeafRight"]
    seen = np.zeros(u, np.int32)
    stack = [(root_gamma, root_hl), (root_gamma + 1, root_hr)]
    while stack:
        c, leaf = stack.pop()
        if leaf:
            seen[c] += 1
        else:
            stack.append((lc[c], hl[c]))
            stack.append((lc[c] + 1, hr[c]))
    return seen


@pytest.mark.parametrize("gen,bits", [("cube", 30), ("scene", 63)])
def test_karras_invariants(oracle, gen, bits):
    x, y, z = synth.uniform_cube(20000, 5) if gen == "cube" else synth.scene(20000, 5)
    st = oracle.build_stages(x, y, z, bits, root_compat=False)
    codes, r = st["codes"], st["radix"]
    u = codes.size
    seen = _subtree_leaves(r, u, r["leftChild"][0], r["hasLeafLeft"][0], r["hasLeafRight"][0])
    assert np.all(seen == 1)
    # prefix check of src/RadixTree.cu:371-381: both children share the node's prefix
    nr = u - 1
    pn = r["prefixN"].astype(np.int64)
    lc = r["leftChild"].astype(np.int64)
    sh = (bits - pn).astype(np.uint64)
    assert np.all((codes[lc] >> sh) == (codes[lc + 1] >> sh))
    # children's prefixes are longer
    for side, flag in ((0, "hasLeafLeft"), (1, "hasLeafRight")):
        inner = r[flag][:nr] == 0
        ch = lc[inner] + side
        assert np.all(pn[ch] > pn[inner])


def test_compat_root_only_changes_node_zero(oracle):
    x, y, z = synth.scene(5000, 6)
    a = oracle.build_stages(x, y, z, 63, root_compat=True)["radix"]
    b = oracle.build_stages(x, y, z, 63, root_compat=False)["radix"]
    for key in ("leftChild", "prefixN", "hasLeafLeft", "hasLeafRight"):
        assert np.array_equal(a[key][1:], b[key][1:])


def test_compat_root_orphans_leaves_in_small_clouds(oracle):
    """src/RadixTree.cu:128-130: with root range l = N-1 some small clouds lose
    a leaf; the full-range root never does."""
    broken = 0
    for s in range(300):
        n = 3 + s % 38
        x, y, z = synth.uniform_cube(n, seed=1000 + s)
        st = oracle.build_stages(x, y, z, 63, root_compat=True)
        u = st["codes"].size
        if u < 3:
            continue
        rc, seen = oracle.octree_check(st["octree"]["nodes"], st["codes"], 63, int(st["radix"]["prefixN"][0] // 3))
        broken += int(not np.all(seen == 1))
        fixed = oracle.build_stages(x, y, z, 63, root_compat=False)
        rc2, seen2 = oracle.octree_check(fixed["octree"]["nodes"], fixed["codes"], 63,
                                         int(fixed["radix"]["prefixN"][0] // 3))
        assert rc2 == 0 and np.all(seen2 == 1)
    assert broken > 0


@pytest.mark.parametrize("gen", ["cube", "scene"])
def test_octree_leaves_once(oracle, gen):
    x, y, z = synth.uniform_cube(30000, 7) if gen == "cube" else synth.scene(30000, 7)
    st = oracle.build_stages(x, y, z, 63, root_compat=False)
    rc, seen = oracle.octree_check(st["octree"]["nodes"], st["codes"], 63, int(st["radix"]["prefixN"][0] // 3))
    assert rc == 0
    assert np.all(seen == 1)
    assert 0.3 < st["octree"]["nodes"].size / st["codes"].size < 0.8


@pytest.mark.parametrize("k", [1, 8, 16, 32])
def test_kdtree_equals_brute(oracle, k):
    x, y, z = synth.scene(6000, 8)
    st = oracle.build_stages(x, y, z)
    p = st["points"]
    a = oracle.knn_exact(p, p[:1500], k)
    b = oracle.knn_exact(p, p[:1500], k, brute=True)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_exact_knn_ties_by_index(oracle):
    g = np.arange(6, dtype=np.float32)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    idx, d2 = oracle.knn_exact(pts, pts, 7)
    for r in range(len(pts)):
        row = list(zip(d2[r], idx[r]))
        assert row == sorted(row)
    # interior point: itself then its 6 face neighbours in index order
    c = 2 * 36 + 2 * 6 + 2
    assert idx[c, 0] == c
    assert sorted(idx[c, 1:]) == list(idx[c, 1:])


def test_fp64_normals_plane_and_orientation(oracle):
    rng = np.random.default_rng(1)
    uv = rng.random((400, 2))
    n = np.array([1.0, 2.0, 2.0]) / 3.0
    a = np.cross(n, [1, 0, 0])
    a /= np.linalg.norm(a)
    b = np.cross(n, a)
    pts = (np.array([3.0, 3.0, 3.0]) + uv[:, :1] * a + uv[:, 1:] * b).astype(np.float32)
    idx, _ = oracle.knn_exact(pts, pts, 10)
    nrm, ev = oracle.normals_f64(pts, idx, pts)
    cos = nrm @ n
    assert np.all(np.abs(np.abs(cos) - 1) < 1e-4)
    # viewpoint (0,0,0) lies on the -n side of the plane: normals point to it
    assert np.all(cos < 0)
    assert np.all(ev[:, 0] <= ev[:, 1] + 1e-18)


def test_compat_search_is_approximate(oracle):
    x, y, z = synth.uniform_cube(30000, 9)
    st = oracle.build_stages(x, y, z)
    p = st["points"]
    q = p[:2000]
    ic, pops = oracle.knn_compat(st["octree"]["nodes"], p, q, 16, want_pops=True)
    ie, _ = oracle.knn_exact(p, q, 16)
    agree = np.mean([set(a) == set(b) for a, b in zip(ic, ie)])
    assert 0.2 < agree < 0.9
    assert pops.mean() > 100


def test_knn_fewer_points_than_k(oracle):
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 2, 0]], np.float32)
    idx, d2 = oracle.knn_exact(pts, pts, 5)
    assert list(idx[0]) == [0, 1, 2, 0, 0]


def test_mlp_grad_modes_agree_to_bf16_rounding(oracle):
    """The oracle's gradient modes (FP64, BF16 forward, BF16 forward with
    BF16 dh as the tensor-core training step) differ only by rounding."""
    rng = np.random.default_rng(4)
    p = rng.normal(0, 0.2, oracle.MLP_PARAMS).astype(np.float32)
    X = rng.uniform(-1, 1, (400, 32)).astype(np.float32)
    y = rng.uniform(-8, 0, 400).astype(np.float32)
    _, l0, g0 = oracle.mlp_grad(p, X, y, round_bf16=False)
    _, l1, g1 = oracle.mlp_grad(p, X, y, round_bf16=True)
    _, l2, g2 = oracle.mlp_grad(p, X, y, round_bf16=2)
    assert l1 == l2  # the forward is the same in both BF16 modes
    assert np.linalg.norm(g2 - g1) / np.linalg.norm(g1) < 1e-2
    assert np.linalg.norm(g1 - g0) / np.linalg.norm(g0) < 5e-2
    assert not np.array_equal(g1, g2)
