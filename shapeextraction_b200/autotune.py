"""Autotuner for the kNN kernel's tile parameters.

Two parameters shape the search kernel's work: `leaf_bucket` (subtrees of at
most this many points are streamed as one tile) and `seed_halo` (Morton-window
points offered on each side of a warp's 32 queries before the tree walk). The
best pair depends on density and k, so it is measured, not guessed: every
candidate is timed on the GPU (CUDA events around the build and the fused kNN
+ normals kernel, median of `reps`) on the caller's own cloud or batch, and the
winner is cached in a JSON file keyed by workload class (size decade, k, code
bits), so that later runs reuse it without re-timing.
"""
from __future__ import annotations

import json
import os
import statistics

import numpy as np

from ._native import Context

CANDIDATES = [(b, h) for b in (32, 64, 96) for h in (8, 16, 32)]
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "shapeextraction_b200", "autotune.json")


def workload_key(n_points: int, k: int, code_bits: int = 63) -> str:
    return f"n1e{int(np.floor(np.log10(max(n_points, 1))))}_k{k}_b{code_bits}"


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(path, table):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _time_cloud(ctx, x, y, z, k, reps):
    times = []
    for _ in range(reps + 1):
        ctx.build(x, y, z)
        ctx.normals(k)
        p = ctx.profile()
        times.append(p["build_ms"]["total"] + p["query_ms"])
    return statistics.median(times[1:])


def tune_cloud(x, y, z, k, code_bits=63, device=0, cache_path=DEFAULT_CACHE, reps=3, force=False):
    """Best (leaf_bucket, seed_halo) for this cloud's class; cached."""
    key = workload_key(len(x), k, code_bits)
    table = _load(cache_path) if cache_path else {}
    if key in table and not force:
        return table[key]
    results = []
    for bucket, halo in CANDIDATES:
        with Context(code_bits=code_bits, device=device, leaf_bucket=bucket, seed_halo=halo) as ctx:
            results.append((_time_cloud(ctx, x, y, z, k, reps), bucket, halo))
    ms, bucket, halo = min(results)
    entry = {"leaf_bucket": bucket, "seed_halo": halo, "ms": ms,
             "timings": [{"leaf_bucket": b, "seed_halo": h, "ms": t} for t, b, h in results]}
    if cache_path:
        table[key] = entry
        _save(cache_path, table)
    return entry


def tune_batch(clouds, ks, code_bits=63, device=0, cache_path=DEFAULT_CACHE, reps=2, force=False):
    """Best (leaf_bucket, seed_halo) for a batch of clouds (se_normals_batch)."""
    sizes = [len(c[0]) for c in clouds]
    key = "batch_" + workload_key(int(np.sum(sizes)), int(np.max(ks)), code_bits) + f"_c{len(clouds)}"
    table = _load(cache_path) if cache_path else {}
    if key in table and not force:
        return table[key]
    results = []
    for bucket, halo in CANDIDATES:
        with Context(code_bits=code_bits, device=device, leaf_bucket=bucket, seed_halo=halo) as ctx:
            import time

            times = []
            for _ in range(reps + 1):
                ctx.synchronize()
                t0 = time.perf_counter()
                ctx.normals_batch(clouds, ks)
                times.append((time.perf_counter() - t0) * 1e3)
            results.append((statistics.median(times[1:]), bucket, halo))
    ms, bucket, halo = min(results)
    entry = {"leaf_bucket": bucket, "seed_halo": halo, "ms": ms,
             "timings": [{"leaf_bucket": b, "seed_halo": h, "ms": t} for t, b, h in results]}
    if cache_path:
        table[key] = entry
        _save(cache_path, table)
    return entry
