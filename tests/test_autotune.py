"""Autotuner (shapeextraction_b200/autotune.py): picks a measured candidate,
caches it per workload class and reuses the cache without timing again."""
import json

import numpy as np
import pytest

from shapeextraction_b200 import autotune, synth


def test_workload_key_classes():
    assert autotune.workload_key(2_000_000, 16) == "n1e6_k16_b63"
    assert autotune.workload_key(999, 8, 30) == "n1e2_k8_b30"
    assert autotune.workload_key(0, 8) == "n1e0_k8_b63"


@pytest.mark.gpu
def test_tune_cloud_and_cache(tmp_path):
    x, y, z = synth.scene(20_000, 5)
    cache = str(tmp_path / "tune.json")
    e = autotune.tune_cloud(x, y, z, 16, cache_path=cache, reps=1)
    assert (e["leaf_bucket"], e["seed_halo"]) in autotune.CANDIDATES
    assert len(e["timings"]) == len(autotune.CANDIDATES)
    assert e["ms"] == min(t["ms"] for t in e["timings"])
    table = json.load(open(cache))
    assert table[autotune.workload_key(x.size, 16)]["leaf_bucket"] == e["leaf_bucket"]
    # a cached class is returned as stored, without timing again
    table[autotune.workload_key(x.size, 16)]["ms"] = -1.0
    json.dump(table, open(cache, "w"))
    assert autotune.tune_cloud(x, y, z, 16, cache_path=cache)["ms"] == -1.0


@pytest.mark.gpu
def test_tune_batch(tmp_path, native):
    """The library's batch tuner returns a tuning in range, leaves it set on
    the context, and the tuned batch gives the same normals as the default."""
    clouds = [synth.scene(n, 40 + i) for i, n in enumerate((3000, 800, 12_000, 70_000))]
    ks = np.array([8, 16, 32, 16], np.int32)
    with native.Context() as ref:
        want, _, _ = ref.normals_batch(clouds, ks)
    with native.Context() as c:
        e = autotune.tune_batch(clouds, ks, cache_path=str(tmp_path / "tb.json"), reps=1, ctx=c)
        assert e["leaf_bucket"] in (48, 64, 96, 128) and e["seed_halo"] in (-1, 8, 16, 32)
        assert e["lanes"] in (4, 8, 16) and e["lane_min_points"] in (32768, 65536, 131072, 262144)
        assert e["blocks_per_sm"] in (0, 2, 3, 4) and e["warps_per_block"] in (0, 2, 4)
        assert e["ms"] > 0
        assert c.batch_tuning() == {k: e[k] for k in native.TUNING_FIELDS}
        got, _, _ = c.normals_batch(clouds, ks)
        np.testing.assert_allclose(np.abs(np.sum(got * want, axis=1)), 1.0, atol=1e-5)
    # cached: the stored entry comes back without timing
    table = json.load(open(tmp_path / "tb.json"))
    key = autotune.batch_key(clouds, ks)
    table[key]["ms"] = -1.0
    json.dump(table, open(tmp_path / "tb.json", "w"))
    assert autotune.tune_batch(clouds, ks, cache_path=str(tmp_path / "tb.json"))["ms"] == -1.0


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [dict(lanes=1, lane_min_points=1000, blocks_per_sm=2, warps_per_block=2),
                                    dict(lanes=16, lane_min_points=300_000, blocks_per_sm=0, warps_per_block=4)])
def test_batch_tunings_give_the_same_normals(native, tuning):
    """Every schedule computes the same thing: lists are exact whatever the
    launch shape, so the normals agree to rounding of the same arithmetic."""
    clouds = [synth.scene(n, 60 + i) for i, n in enumerate((2000, 500, 40_000, 90_000, 7000))]
    ks = np.array([16, 8, 32, 16, 10], np.int32)
    with native.Context() as ref:
        want, _, u0 = ref.normals_batch(clouds, ks)
    with native.Context() as c:
        c.set_batch_tuning({**c.batch_tuning(), **tuning})
        got, _, u1 = c.normals_batch(clouds, ks)
    assert np.array_equal(u0, u1)
    assert np.array_equal(got, want)
