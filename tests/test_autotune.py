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
def test_tune_batch(tmp_path):
    clouds = [synth.scene(n, 40 + i) for i, n in enumerate((3000, 800, 12_000))]
    ks = np.array([8, 16, 32], np.int32)
    e = autotune.tune_batch(clouds, ks, cache_path=str(tmp_path / "tb.json"), reps=1)
    assert (e["leaf_bucket"], e["seed_halo"]) in autotune.CANDIDATES
