"""Learned search-radius proposal: oracle self-check (CPU), GPU forward and
backward kernels against the CPU oracle, tensor-core inference against the
training forward, training on a held-out cloud, exactness of the learned
search (including forced misses), and what the model gains over the plain
search (work counters)."""
import numpy as np
import pytest

from shapeextraction_b200 import learned, synth


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(6337, np.float32)
    p[:2048] = rng.uniform(-0.4, 0.4, 2048)
    p[2048:2112] = rng.uniform(-0.1, 0.1, 64)
    p[2112:6208] = rng.uniform(-0.3, 0.3, 4096)
    p[6208:6272] = rng.uniform(-0.1, 0.1, 64)
    p[6272:6336] = rng.uniform(-0.3, 0.3, 64)
    p[6336] = -3.0
    return p


def test_oracle_mlp_grad_finite_differences(oracle):
    """Backward formulas of the oracle vs central differences (plain double math)."""
    rng = np.random.default_rng(0)
    p = _rand_params(1)
    X = rng.uniform(-1, 1, (40, 32)).astype(np.float32)
    y = rng.uniform(-5, 0, 40).astype(np.float32)
    _, loss, g = oracle.mlp_grad(p, X, y, round_bf16=False)
    for i in list(range(0, 2048, 97)) + list(range(2048, 6337, 131)) + [6336]:
        h = 1e-2 * max(abs(float(p[i])), 1e-2)
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (oracle.mlp_grad(pp, X, y, round_bf16=False)[1] - oracle.mlp_grad(pm, X, y, round_bf16=False)[1]) / (
            float(pp[i]) - float(pm[i]))
        assert abs(fd - g[i]) <= 1e-3 * max(1.0, abs(g[i])), (i, fd, g[i])


@pytest.mark.gpu
def test_gpu_forward_and_grad_match_oracle(native, oracle):
    rng = np.random.default_rng(2)
    p = _rand_params(3)
    X = rng.uniform(-1, 1, (3000, 32)).astype(np.float32)
    y = rng.uniform(-8, 0, 3000).astype(np.float32)
    with native.Context() as c:
        c.mlp_params(p)
        yh = c.mlp_forward(X)
        loss, g = c.mlp_grad(X, y)
    yo, lo, go = oracle.mlp_grad(p, X, y, round_bf16=True)
    assert np.array_equal(yh.astype(np.float64), yo)  # same roundings, same fmaf order
    # The gradient comes from the tensor-core training step: its FP32 sums run
    # in the mma order (an activation can round to the neighbouring BF16
    # value), and dh1, dh2 enter the products in BF16, which the oracle's mode
    # 2 restates.
    _, lo2, go2 = oracle.mlp_grad(p, X, y, round_bf16=2)
    assert abs(loss - lo2) <= 1e-4 * abs(lo2)
    rel = np.linalg.norm(g - go2) / np.linalg.norm(go2)
    assert rel < 2e-3, rel
    big = np.abs(go2) > 1e-2 * np.abs(go2).max()
    assert np.max(np.abs(g[big] - go2[big]) / np.abs(go2[big])) < 2e-2
    # and it stays close to the gradient without the BF16 rounding of dh
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 1e-2


@pytest.mark.gpu
def test_pinball_gradient_matches_oracle(native, oracle):
    """The quantile (pinball) loss of se_mlp_set_loss, against the oracle's
    restatement with the same roundings."""
    rng = np.random.default_rng(6)
    p = _rand_params(4)
    X = rng.uniform(-1, 1, (3000, 32)).astype(np.float32)
    y = rng.uniform(-8, 0, 3000).astype(np.float32)
    with native.Context() as c:
        c.mlp_params(p)
        c.mlp_set_loss(0.9)
        loss, g = c.mlp_grad(X, y)
        with pytest.raises(native.ShapexError):
            c.mlp_set_loss(1.0)
    _, lo, go = oracle.mlp_grad(p, X, y, round_bf16=2, quantile=0.9)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 2e-3


@pytest.mark.gpu
def test_tensor_core_inference_matches_training_forward(native):
    x, y, z = synth.scene(50_000, 5)
    with native.Context() as c:
        c.build(x, y, z)
        c.mlp_init(7)
        X = c.features()
        assert X.shape == (c.info()["n_points"], 32) and np.all(np.isfinite(X))
        yf = c.mlp_forward(X)
        yt, r2 = c.mlp_predict()
        assert np.max(np.abs(yt - yf)) < 2e-2 * max(1.0, np.abs(yf).max())
        assert np.all(r2 > 0)


@pytest.fixture(scope="module")
def trained(native):
    """A model trained on a held-out cloud (seed 101)."""
    from shapeextraction_b200 import learned

    x, y, z = synth.scene(300_000, 101)
    c = native.Context()
    c.build(x, y, z)
    rep = learned.train_radius_model(c, 16, steps=800, batch=8192, lr=2e-3, seed=0)
    yield c, rep
    c.close()


@pytest.mark.gpu
def test_training_converges(trained):
    c, rep = trained
    L = rep["losses"]
    # the scene's surface density is nearly uniform, so the target variance is
    # small to begin with; the model must still remove a clear share of it
    assert L[-50:].mean() < 0.7 * L[:20].mean()
    assert rep["residual_std"] < 1.0  # in log2(r^2) units


@pytest.mark.gpu
def test_learned_search_exact_and_gain(native, oracle, trained):
    from shapeextraction_b200 import learned

    src, rep = trained
    x, y, z = synth.scene(300_000, 1)  # evaluation cloud: same generator and size, another seed
    with native.Context() as c:
        c.build(x, y, z)
        learned.transfer(src, c, rep["margin"])
        pts = c.points()
        plain_idx, plain_d2 = c.knn_self(16, with_d2=True)
        plain_n = c.normals(16)
        s_plain = c.stats()
        for skip in (False, True):
            c.set_learned(True, skip_seed=skip)
            idx, d2 = c.knn_self(16, with_d2=True)
            assert np.array_equal(idx, plain_idx) and np.array_equal(d2, plain_d2)
            nrm = c.normals(16)
            assert np.array_equal(nrm, plain_n)
            s = c.stats()
            assert s["learned_misses"] < 0.05 * pts.shape[0]
            assert s["candidates"] < s_plain["candidates"]  # tighter starting bound
            assert s["cell_warps"] == 0 and s["cell_fallbacks"] == 0  # the capped tree walk
        ei, ed = oracle.knn_exact(pts, pts[:20000], 16)
        assert np.array_equal(plain_idx[:20000], ei)
    # the cell scan (the learned attempt without a tree walk) gives the same lists
    with native.Context(learned_cell_scan=True) as c:
        c.build(x, y, z)
        learned.transfer(src, c, rep["margin"])
        c.set_learned(True, skip_seed=True)
        idx, d2 = c.knn_self(16, with_d2=True)
        assert np.array_equal(idx, plain_idx) and np.array_equal(d2, plain_d2)
        assert np.array_equal(c.normals(16), plain_n)
        s = c.stats()
        warps = (pts.shape[0] + 31) // 32
        assert s["cell_warps"] > 0.9 * warps, s
        assert s["cell_warps"] + s["cell_fallbacks"] == warps


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 5, 8, 10, 12, 16, 20, 32])
def test_cell_scan_exact_on_lattice_ties(native, oracle, trained, k):
    """Integer lattice with repeated points (many equal distances): the cell
    scan offers candidates in another order than the walk, and the lists must
    still equal the oracle's, ties broken by index. Every k's kernel runs the
    cell scan (the model's bounds are per-cloud, so calibration does not
    matter for exactness)."""
    src, rep = trained
    rng = np.random.default_rng(5)
    x, y, z = (rng.integers(0, 40, 80_000).astype(np.float32) for _ in range(3))
    with native.Context(learned_cell_scan=True) as c:
        c.build(x, y, z)
        learned.transfer(src, c, rep["margin"])
        pts = c.points()
        c.set_learned(True, skip_seed=True)
        idx, d2 = c.knn_self(k, with_d2=True)
        ei, ed = oracle.knn_exact(pts, pts, k)
        assert np.array_equal(d2, ed)
        assert np.array_equal(idx, ei)
        assert c.stats()["cell_warps"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("margin", [6.0, 40.0])
def test_cell_scan_oversized_caps_fall_back_exactly(native, oracle, trained, margin):
    """Caps far too large: the warps' cells hold more points than a cell scan
    takes (or span the whole cube), so the learned attempt walks the tree with
    the cap instead; results stay exact."""
    src, rep = trained
    x, y, z = synth.scene(60_000, 3)
    with native.Context(learned_cell_scan=True) as c:
        c.build(x, y, z)
        c.mlp_params(src.mlp_params())
        c.mlp_set_margin(margin)
        c.set_learned(True, skip_seed=True)
        idx, d2 = c.knn_self(16, with_d2=True)
        s = c.stats()
        assert s["cell_fallbacks"] > 0, s
        pts = c.points()
        ei, ed = oracle.knn_exact(pts, pts, 16)
        assert np.array_equal(idx, ei) and np.array_equal(d2, ed)


@pytest.mark.gpu
def test_learned_forced_misses_fall_back(native, oracle, trained):
    src, rep = trained
    x, y, z = synth.scene(60_000, 2)
    with native.Context() as c:
        c.build(x, y, z)
        c.mlp_params(src.mlp_params())
        c.mlp_set_margin(-12.0)  # bounds far too small: every query misses
        pts = c.points()
        ei, _ = oracle.knn_exact(pts, pts, 16)
        for skip in (False, True):  # the capped walk with and without the seed
            c.set_learned(True, skip_seed=skip)
            idx = c.knn_self(16)
            assert c.stats()["learned_misses"] == c.info()["n_points"]
            assert np.array_equal(idx, ei)
    with native.Context(learned_cell_scan=True) as c:  # the cell scan
        c.build(x, y, z)
        c.mlp_params(src.mlp_params())
        c.mlp_set_margin(-12.0)
        c.set_learned(True, skip_seed=True)
        assert np.array_equal(c.knn_self(16), ei)
        assert c.stats()["learned_misses"] == c.info()["n_points"]


@pytest.mark.gpu
def test_model_save_load(native, trained, tmp_path):
    src, rep = trained
    f = str(tmp_path / "radius.sxmlp")
    src.mlp_save(f)
    with native.Context() as c:
        c.mlp_load(f)
        assert np.array_equal(c.mlp_params(), src.mlp_params())
