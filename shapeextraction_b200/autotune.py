"""Autotuner for the kNN kernel's tile parameters and the batch schedule.

Two parameters shape the search kernel's work: `leaf_bucket` (subtrees of at
most this many points are streamed as one tile) and `seed_halo` (Morton-window
points offered on each side of a warp's 32 queries before the tree walk). The
batched path adds its schedule: stream lanes, the size above which a cloud is
queried on its lane, and the persistent launches' resident blocks per SM and
warps per block. The best values depend on density, k and the batch's size
mix, so they are measured, not guessed, on the caller's own cloud or batch
(single clouds here with CUDA events around the build and the fused kNN +
normals kernel; batches in the library, se_tune_batch), and the winner is
cached in a JSON file keyed by workload class (size decade, k, code bits,
cloud count), so that later runs reuse it without re-timing.
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


def batch_key(clouds, ks, code_bits=63) -> str:
    """Class of a batch given as normals_batch takes it: a list of (x, y, z)
    clouds, or concatenated (x, y, z) with ks=(ks, offsets)."""
    if isinstance(ks, tuple):
        ks, offsets = ks
        total, n = int(offsets[-1]), len(ks)
    else:
        total, n = int(np.sum([len(c[0]) for c in clouds])), len(clouds)
    return "batch_" + workload_key(total, int(np.max(ks)), code_bits) + f"_c{n}"


def tune_batch(clouds, ks, code_bits=63, device=0, cache_path=DEFAULT_CACHE, reps=2, force=False, ctx=None):
    """Best se_normals_batch tuning for this batch's class: bucket size, seed
    halo, stream lanes, the per-lane query cut-off, and the persistent
    launches' resident blocks and block shape. The search runs in the library
    (se_tune_batch: CUDA events around whole batched calls, one parameter at
    a time over two rounds); the winner is cached per class and, when `ctx`
    is given, left set on it."""
    key = batch_key(clouds, ks, code_bits)
    table = _load(cache_path) if cache_path else {}
    if key in table and not force:
        entry = table[key]
    else:
        own = ctx is None
        c = Context(code_bits=code_bits, device=device) if own else ctx
        try:
            entry = c.tune_batch(clouds, ks, reps=reps)
        finally:
            if own:
                c.close()
        if cache_path:
            table[key] = entry
            _save(cache_path, table)
    if ctx is not None:
        ctx.set_batch_tuning(entry)
    return entry
