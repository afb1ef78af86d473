#!/usr/bin/env python
"""Benchmark of the normal-estimation path: normals/s end to end at k=16.

Workload (default): precision_20M_k16, 20M points of the precision mix
(sphere/plane scene surfaces, planes with anisotropic noise of sigma 1e-5 to
1e-2, collinear segments, 1e-4-scale clusters offset by 1e3), 63-bit Morton
codes, k=16, exact kNN, FP64 eigensolve below a relative eigengap of 1e-6.
Other workloads (--workload): scene_2M_k16, gmm_50M_k16, cube_100k_k10,
batch_256.

A step is one pass of the path over one cloud: build (bbox, encode, sort,
dedup, radix tree, octree) followed by normals for every unique point.
  value  device-resident: inputs already in HBM, normals written to HBM
  e2e    through the C ABI with host buffers: pinned host x/y/z copied in and
         the normals copied out inside the timed region
  e2e_pipelined  the e2e steps on two contexts driven by two host threads,
         so that one step's input copy overlaps the other's build and search
Both are timed with CUDA events on the stream the library runs on, L2 flushed
(256 MB write) before every timed step, max over ranks. The learned-radius
pipeline is the headline; the plain path is timed beside it, and the
reference's own CUDA build (oracle/_ref/refdriver, when it was compiled) runs
on the same cloud, host in to host out.

  python bench.py [--gpus N --steps K --warmup W] [--mode replicas|sharded]
                  [--impl reference]

--gpus N > 1 without a launcher re-runs this script under
torch.distributed.run with N ranks, one per GPU. --mode replicas (default):
every rank runs an independent replica on its own cloud (weak scaling; the
path has no exchange step). --mode sharded: one cloud, broadcast from rank 0,
built on every rank, queries split into contiguous ranges, normals
all-gathered (strong scaling). `--impl reference` times the reference
pipeline restated on the host cores (rank 0 only), and the reference's own
CUDA build when it was compiled (oracle/_ref).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "normals/sec end-to-end @k=16: learned-radius vs plain GPU, exact kNN, ≤1e-3 rad"


def _workloads(points=None):
    """The configurations' workloads; `points` resizes the single-cloud ones
    (for profiling runs on a smaller or larger cloud of the same generator)."""
    from shapeextraction_b200 import synth

    wl = _workload_table(synth)
    if points:
        for key, w in wl.items():
            if not w.get("batched"):
                w["gen"] = (lambda g: (lambda s: g(int(points), s)))(w["sample"])
                w["desc"] = f"{w['desc']} (resized to {int(points)} points)"
    return wl


def _workload_table(synth):
    return {
        "scene_2M_k16": dict(gen=lambda s: synth.scene(2_000_000, s), sample=synth.scene, k=16, code_bits=63,
                             desc="2M points on 32 spheres + 8 planes, jitter 0.002, 63-bit codes, k=16"),
        "precision_20M_k16": dict(gen=lambda s: synth.precision_mix(20_000_000, s), sample=synth.precision_mix, k=16,
                                  code_bits=63, eigengap=1e-6,
                                  desc="20M points precision mix, 63-bit codes, k=16, FP64 eigensolve below a "
                                       "relative eigengap of 1e-6"),
        "gmm_50M_k16": dict(gen=lambda s: synth.gaussian_mixture(50_000_000, s), sample=synth.gaussian_mixture, k=16,
                            code_bits=63,
                            desc="50M points Gaussian mixture + surfaces, 63-bit codes, k=16"),
        "cube_100k_k10": dict(gen=lambda s: synth.uniform_cube(100_000, s), sample=synth.uniform_cube, k=10,
                              code_bits=30,
                              desc="100k uniform points, 30-bit codes, k=10"),
        "batch_256": dict(gen=lambda s: synth.batched_clouds(256, s), sample=synth.scene, k=None, code_bits=63,
                          batched=True,
                          desc="256 independent scenes, sizes log-uniform in [1k, 500k], k per cloud in {8,16,32}, "
                               "one se_normals_batch call"),
    }


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_field(workload, field):
    """A number from the committed ncu summary of the fused kNN kernel
    (profiles/knn_normals_<workload>.md), given there as `field: value`."""
    p = os.path.join(ROOT, "profiles", f"knn_normals_{workload}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(field + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def knn_roofline(u, m, k, q_ms, workload, clocks, num_sms):
    """Roofline object of the fused kNN + normals kernel.

    HBM: algorithmic bytes per launch are the compulsory traffic of the kNN +
    normal row of the path's byte model, 12u query points + 12u neighbour
    points + 32m octree nodes read, 12u normals + 4ku neighbour indices
    written: 36u + 32m + 4ku. The fused kernel never writes the indices (the
    normals are computed from the lists in registers), so the 4ku term is
    bytes it saves, counted as the model counts them.
    Issue: warp instructions per launch (the committed ncu figure per query,
    times u) over the issue capacity of the launch, num_sms x 4 schedulers x
    the median SM clock sampled during the timed region x the launch time.
    This kernel is bound by instruction issue, not by HBM."""
    alg = 36 * u + 32 * m + 4 * k * u
    peak, peak_kind = _peaks()
    achieved = alg / (q_ms * 1e-3) / 1e9
    traffic_pq = _profile_field(workload, "traffic_bytes_per_query")
    out = {"bound": "hbm", "kernel": "k_knn (fused kNN + covariance + eigensolve + orientation)",
           "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
           "traffic": None if traffic_pq is None else traffic_pq * u,
           "alg_bytes_per_launch": int(alg),
           "definition": "alg = 36u + 32m + 4ku bytes (12u queries + 12u neighbour points + 32m octree nodes read, "
                         "12u normals + 4ku indices written; the fused kernel writes no indices) / CUDA-event "
                         "launch time; traffic = ncu dram read+write bytes per query of this workload x u",
           "launch_ms": q_ms}
    ipq = _profile_field(workload, "warp_instructions_per_query")
    mhz = (clocks or {}).get("sm_mhz")
    if ipq is not None and mhz:
        instr = ipq * u
        cap = num_sms * 4 * mhz * 1e6 * q_ms * 1e-3
        out["issue"] = {"warp_instructions_per_launch": instr, "issue_capacity": cap, "frac": instr / cap,
                        "sm_mhz": mhz, "definition": "ncu warp instructions per query x u / (SMs x 4 schedulers "
                                                     "x median SM clock x launch time)"}
    return out


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [c.strip() for c in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i in range(4) if r[i].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _init_dist(world, local, backend="nccl", single=False):
    """One process group per run, short timeout (ranks that wait on each
    other end with an error instead of hanging). single: a one-rank group
    too (the sharded path calls the collectives whatever the rank count)."""
    if world <= 1 and not single:
        return
    if world <= 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", str(_free_port()))
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    if backend == "nccl":
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=timedelta(seconds=120))


def _reduce(vals, op, device):
    """Elementwise max or sum of a list of floats over all ranks."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return list(vals)
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def run_ours(a):
    import torch
    import torch.distributed as dist

    from shapeextraction_b200 import Context
    from shapeextraction_b200.distributed import shard_ranges, sharded_normals

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    sharded = a.mode == "sharded"
    _init_dist(world, local, single=sharded)
    dev = torch.device("cuda", local)
    wl = _workloads(a.points)[a.workload]
    k = wl["k"]
    # replicas: one cloud per rank; sharded: rank 0's cloud, broadcast each step
    x, y, z = wl["gen"](a.seed + (0 if sharded else rank))
    n = x.size
    hx, hy, hz = (torch.from_numpy(v).pin_memory() for v in (x, y, z))
    dx, dy, dz = (v.cuda() for v in (hx, hy, hz))
    stream = torch.cuda.current_stream()
    ctx = Context(code_bits=wl["code_bits"], device=local, stream=stream.cuda_stream,
                  eigengap_fp64=a.eigengap, leaf_bucket=a.bucket, seed_halo=a.halo)
    u = ctx.build(dx, dy, dz)["n_points"]
    out_dev = torch.empty((u, 3), dtype=torch.float32, device="cuda")
    out_host = torch.empty((u, 3), dtype=torch.float32).pin_memory()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    if sharded:
        q_start, q_count = shard_ranges(u, world)[rank]
    else:
        q_start, q_count = 0, u

    if sharded:
        # the whole sharded call: broadcast of rank 0's input, redundant
        # build, this rank's range, all-gather of every range's normals
        def step_device():
            return sharded_normals(ctx, dx if rank == 0 else None, dy if rank == 0 else None,
                                   dz if rank == 0 else None, k)

        def step_e2e():
            # rank 0 copies its pinned host input in (inside the broadcast) and
            # reads the gathered normals back to pinned host memory
            res = sharded_normals(ctx, hx if rank == 0 else None, hy if rank == 0 else None,
                                  hz if rank == 0 else None, k)
            if rank == 0:
                out_host.copy_(res, non_blocking=True)
            return res
    else:
        def step_device():
            ctx.build(dx, dy, dz)
            ctx.normals(k, out=out_dev)

        def step_e2e():
            ctx.build(hx, hy, hz)
            ctx.normals(k, out=out_host)

    def timed(step, steps, prof=None):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
            if prof is not None:
                prof.append(ctx.profile())
        torch.cuda.synchronize()
        return sum(s.elapsed_time(e) for s, e in ev)

    # a second context on its own stream for the pipelined end-to-end figure:
    # two host threads each run whole steps through the C ABI (pinned input
    # copied in, normals written to pinned host memory) on their own context,
    # so one step's input copy overlaps the other's search
    ctx2 = stream2 = out_host2 = None
    if not sharded:
        stream2 = torch.cuda.Stream(device=dev)
        ctx2 = Context(code_bits=wl["code_bits"], device=local, stream=stream2.cuda_stream,
                       eigengap_fp64=a.eigengap, leaf_bucket=a.bucket, seed_halo=a.halo)
        out_host2 = torch.empty((u, 3), dtype=torch.float32).pin_memory()

    def timed_pipelined(steps):
        import threading

        ctxs, outs, streams = (ctx, ctx2), (out_host, out_host2), (stream, stream2)
        start = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        start.record(stream)
        stream2.wait_event(start)
        errs = []

        def run(t):
            try:
                torch.cuda.set_device(local)
                for _ in range(t, steps, 2):
                    ctxs[t].build(hx, hy, hz)
                    ctxs[t].normals(k, out=outs[t])
                ends[t].record(streams[t])
            except BaseException as e:  # re-raised on the main thread
                errs.append(e)

        th = [threading.Thread(target=run, args=(t,)) for t in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errs:
            raise errs[0]
        torch.cuda.synchronize()
        return max(start.elapsed_time(e) for e in ends)

    def measure():
        # the clock sampler starts before the warm-up so that its first
        # samples (nvidia-smi needs a moment to start) fall under load
        clk = Clocks(local)
        clk.start()
        for _ in range(a.warmup):
            step_device()
            step_e2e()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        profs = []
        ms_dev = timed(step_device, a.steps, profs)
        stats = ctx.stats()
        ms_e2e = timed(step_e2e, a.steps)
        ms_pipe = 0.0
        if ctx2 is not None:
            timed_pipelined(2)  # warm-up: the second context's first build allocates
            ms_pipe = timed_pipelined(a.steps)
        clocks = clk.stop()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms_dev, ms_e2e, ms_pipe = _reduce([ms_dev, ms_e2e, ms_pipe], "max", dev)
        return {"ms_dev": ms_dev, "ms_e2e": ms_e2e, "ms_pipe": ms_pipe, "profs": profs, "stats": stats,
                "clocks": clocks}

    # normals per step over all ranks: every rank's cloud (replicas) or the one cloud (sharded)
    u_all = u if sharded else int(_reduce([u], "sum", dev)[0])

    plain = None if (a.skip_plain and not a.no_learned) else measure()
    lrn = None
    if not a.no_learned:
        from shapeextraction_b200 import learned

        # train on a held-out cloud of the same generator and size (another seed)
        xt, yt, zt = wl["gen"](101 + rank)
        t0 = time.perf_counter()
        ctx.build(xt, yt, zt)
        rep = learned.train_radius_model(ctx, k, steps=a.train_steps, batch=8192, lr=2e-3, seed=rank)
        train_s = time.perf_counter() - t0
        del xt, yt, zt
        ctx.build(dx, dy, dz)
        ctx.set_learned(True, skip_seed=not a.learned_keep_seed)
        if ctx2 is not None:
            with tempfile.TemporaryDirectory() as td:
                ctx.mlp_save(os.path.join(td, "radius.mlp"))
                ctx2.mlp_load(os.path.join(td, "radius.mlp"))
            ctx2.set_learned(True, skip_seed=not a.learned_keep_seed)
        lrn = measure()
        ctx.set_learned(False)
        if ctx2 is not None:
            ctx2.set_learned(False)
        lrn["train"] = {"seconds_incl_features_and_targets": train_s, "steps": a.train_steps,
                        "final_loss": float(rep["losses"][-20:].mean()), "first_loss": float(rep["losses"][:20].mean()),
                        "margin_log2": rep["margin"], "residual_std": rep["residual_std"],
                        "held_out_seed": 101 + rank}
    compat = None
    if not a.no_compat and not sharded:
        # the reference's own search and covariance, bit-identical neighbour
        # lists, on the GPU (device-resident inputs, same flush between steps)
        with Context(code_bits=wl["code_bits"], device=local, stream=stream.cuda_stream, search_compat=True) as cc:
            out_c = torch.empty((u, 3), dtype=torch.float32, device="cuda")

            def step_compat():
                cc.build(dx, dy, dz)
                cc.normals(k, out=out_c)

            for _ in range(a.compat_warmup):
                step_compat()
            n_c = max(1, a.compat_steps)
            cprofs = []
            evs = []
            for i in range(n_c):
                flush.fill_(float(i))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step_compat()
                e1.record(stream)
                evs.append((e0, e1))
                cprofs.append(cc.profile())
            torch.cuda.synchronize()
            ms_c = _reduce([sum(e0.elapsed_time(e1) for e0, e1 in evs)], "max", dev)[0]
            compat = {"value": u_all * n_c / (ms_c * 1e-3), "ms_per_step": ms_c / n_c, "steps": n_c,
                      "knn_normals_ms": statistics.mean(p["query_ms"] for p in cprofs),
                      "desc": "reference search (face-plane box distance, 32-slot node heap) and FP32 "
                              "covariance, neighbour lists identical to the reference build's; one GPU per replica"}
    head = lrn if lrn is not None else plain
    ms_dev, ms_e2e, profs, stats, clocks = head["ms_dev"], head["ms_e2e"], head["profs"], head["stats"], head["clocks"]

    # dominant kernel: the fused kNN + normals kernel (this rank's range)
    q_ms = statistics.mean(p["query_ms"] for p in profs)
    build_ms = {s: statistics.mean(p["build_ms"][s] for p in profs) for s in profs[0]["build_ms"]}
    launches = sum(p["build_launches"] + p["query_launches"] for p in profs)
    m = ctx.info()["n_octree"]
    num_sms = torch.cuda.get_device_properties(local).multi_processor_count
    roof = knn_roofline(q_count, m, k, q_ms, a.workload, clocks, num_sms)
    # whole step: B_alg = 72n + (96 + 4k)u + 64m bytes over the device step time
    b_step = 72 * n + (96 + 4 * k) * u + 64 * m
    peak, _ = _peaks()
    step_roof = {"alg_bytes_per_step": int(b_step), "achieved": b_step / (ms_dev / a.steps * 1e-3) / 1e9,
                 "frac": b_step / (ms_dev / a.steps * 1e-3) / 1e9 / peak,
                 "definition": "72n + (96 + 4k)u + 64m bytes (every stage reads its inputs once and writes its "
                               "outputs once) / device step time, against the same HBM peak"}

    cpu = None
    ref_cuda = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a.workload, a.seed, a.cpu_sample)
    if rank == 0 and world == 1 and not a.no_reference_cuda:
        ref_cuda = reference_cuda(a.workload, a.seed, xyz=(x, y, z))

    if rank == 0:
        e2e_value = u_all * a.steps / (ms_e2e * 1e-3)
        line = {
            "metric": METRIC,
            "value": u_all * a.steps / (ms_dev * 1e-3),
            "unit": "normals/s",
            "n_gpus": world,
            "steps": a.steps,
            "warmup": a.warmup,
            "ms_per_step": ms_dev / a.steps,
            "higher_is_better": True,
            "scaling": "strong" if sharded else "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": a.workload, "desc": wl["desc"], "n_points": int(n), "unique_points": int(u),
                       "k": k, "code_bits": wl["code_bits"], "octree_nodes": int(m),
                       "l2": "flushed by a 256 MB device write before every timed step",
                       "mode": a.mode,
                       "parallelism": (f"query-sharded over {world} rank(s): broadcast input, redundant build, "
                                       f"contiguous query ranges, all-gather of normals") if sharded else
                                      f"{world} independent replica(s), one cloud per GPU",
                       "leaf_bucket": a.bucket, "seed_halo": a.halo if a.halo >= 0 else (32 if k > 16 else 16),
                       "eigengap_fp64": a.eigengap},
            "e2e": {"value": e2e_value, "unit": "normals/s",
                    "ms_per_step": ms_e2e / a.steps, "h2d_bytes_per_step": int(12 * n),
                    "d2h_bytes_per_step": int(12 * u)},
            "e2e_pipelined": None if not head["ms_pipe"] else {
                "value": u_all * a.steps / (head["ms_pipe"] * 1e-3), "unit": "normals/s",
                "ms_per_step": head["ms_pipe"] / a.steps, "h2d_bytes_per_step": int(12 * n),
                "d2h_bytes_per_step": int(12 * u),
                "definition": "the same steps through the C ABI on two contexts and streams, driven by two host "
                              "threads (step i on context i mod 2): one step's input copy overlaps the other's "
                              "build and search; CUDA events from before the first copy to the last normals; no "
                              f"L2 flush between steps: each step copies its input ({12 * n / 1e6:.0f} MB) in "
                              "from the host" + (", more than the 126 MB L2" if 12 * n > 126e6 else "")},
            "roofline": roof,
            "step_roofline": step_roof,
            "pipeline": "learned-radius" if lrn is not None else "plain",
            "plain": None if plain is None else {
                "value": u_all * a.steps / (plain["ms_dev"] * 1e-3), "ms_per_step": plain["ms_dev"] / a.steps,
                "e2e_value": u_all * a.steps / (plain["ms_e2e"] * 1e-3),
                "knn_normals_ms": statistics.mean(p["query_ms"] for p in plain["profs"]),
                "search_per_warp": {key: plain["stats"][key] / max(q_count / 32, 1) for key in
                                    ("nodes_visited", "buckets_scanned", "merge_steps")},
                "search_per_query": {key: plain["stats"][key] / max(q_count, 1) for key in
                                     ("candidates", "inserts")}},
            "learned": None if lrn is None else {
                "value": u_all * a.steps / (lrn["ms_dev"] * 1e-3), "ms_per_step": lrn["ms_dev"] / a.steps,
                "e2e_value": u_all * a.steps / (lrn["ms_e2e"] * 1e-3),
                "knn_normals_ms": statistics.mean(p["query_ms"] for p in lrn["profs"]),
                "misses_per_query": lrn["stats"]["learned_misses"] / max(q_count, 1),
                "skip_seed": not a.learned_keep_seed, **lrn["train"]},
            "learned_over_plain": None if (lrn is None or plain is None) else {
                "device": plain["ms_dev"] / lrn["ms_dev"], "e2e": plain["ms_e2e"] / lrn["ms_e2e"],
                "knn_normals": (statistics.mean(p["query_ms"] for p in plain["profs"]) /
                                statistics.mean(p["query_ms"] for p in lrn["profs"]))},
            "compat": compat,
            "stages_ms": {**build_ms, "knn_normals": q_ms},
            "gpu_launches": int(launches),
            "fp64_solves_last_step": stats["fp64_solves"],
            "search_per_warp": {key: stats[key] / max(q_count / 32, 1) for key in
                                ("nodes_visited", "buckets_scanned", "merge_steps", "cell_warps",
                                 "cell_fallbacks")},
            "search_per_query": {key: stats[key] / max(q_count, 1) for key in ("candidates", "inserts")},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "reference_cuda_build": ref_cuda,
            "vs_reference_cuda": (e2e_value / ref_cuda["value"]) if ref_cuda and "value" in ref_cuda else None,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ctx2 is not None:
        ctx2.close()
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


def run_batch(a):
    import torch
    import torch.distributed as dist

    from shapeextraction_b200 import Context, autotune

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    _init_dist(world, local)
    wl = _workloads()[a.workload]
    clouds, ks = wl["gen"](a.seed + rank)
    ks = np.ascontiguousarray(ks, np.int32)
    sizes = np.array([len(c[0]) for c in clouds], np.int64)
    offsets = np.zeros(len(clouds) + 1, np.int64)
    offsets[1:] = np.cumsum(sizes)
    total = int(offsets[-1])
    host = [torch.from_numpy(np.ascontiguousarray(np.concatenate([c[i] for c in clouds]), np.float32)).pin_memory()
            for i in range(3)]
    dev = [h.cuda() for h in host]
    stream = torch.cuda.current_stream()
    ctx = Context(code_bits=wl["code_bits"], device=local, stream=stream.cuda_stream, eigengap_fp64=a.eigengap,
                  leaf_bucket=a.bucket, seed_halo=a.halo)
    tuning = None
    if a.autotune:
        # the library's tuner on this batch (device-resident inputs), cached per class, set on ctx
        tuning = autotune.tune_batch(tuple(dev), (ks, offsets), code_bits=wl["code_bits"], device=local,
                                     cache_path=a.autotune_cache, ctx=ctx)
    bucket, halo = ctx.batch_tuning()["leaf_bucket"], ctx.batch_tuning()["seed_halo"]
    out_dev = torch.empty((total, 3), dtype=torch.float32, device="cuda")
    out_host = torch.empty((total, 3), dtype=torch.float32).pin_memory()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    _, _, u = ctx.normals_batch(tuple(dev), (ks, offsets), out=out_dev)
    u_sum = int(u.sum())

    def timed(step, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return sum(s.elapsed_time(e) for s, e in ev)

    step_dev = lambda: ctx.normals_batch(tuple(dev), (ks, offsets), out=out_dev)  # noqa: E731
    step_e2e = lambda: ctx.normals_batch(tuple(host), (ks, offsets), out=out_host)  # noqa: E731
    clk = Clocks(local)
    clk.start()
    for _ in range(a.warmup):
        step_dev()
        step_e2e()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms_dev = timed(step_dev, a.steps)
    ms_e2e = timed(step_e2e, a.steps)
    clocks = clk.stop()
    prof = ctx.profile()
    # per step: the build and query kernels of every cloud, the e2e arm's too
    launches = 2 * a.steps * (prof["build_launches"] + prof["query_launches"])
    if world > 1:
        t = torch.tensor([ms_dev, ms_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_dev, ms_e2e = float(t[0]), float(t[1])
        tu = torch.tensor([u_sum], dtype=torch.int64, device="cuda")
        dist.all_reduce(tu, op=dist.ReduceOp.SUM)
        u_all = int(tu[0])
    else:
        u_all = u_sum
    # whole-pipeline algorithmic bytes (bbox, encode, sort, dedup, tree, search, normals; no octree)
    alg = float(np.sum(72 * sizes + (96 + 4 * ks.astype(np.int64)) * u))
    peak, peak_kind = _peaks()
    achieved = alg / (ms_dev / a.steps * 1e-3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a.workload, a.seed, a.cpu_sample)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": u_all * a.steps / (ms_dev * 1e-3), "unit": "normals/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_dev / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
            "pipeline": "plain (batched)",
            "config": {"workload": a.workload, "desc": wl["desc"], "clouds": len(clouds), "n_points": total,
                       "unique_points": u_sum, "k_counts": {str(k): int((ks == k).sum()) for k in (8, 16, 32)},
                       "leaf_bucket": bucket,
                       "seed_halo": halo if halo >= 0 else "per k: 16 up to k=16, 32 above", "autotune": tuning,
                       "batch_tuning": ctx.batch_tuning(),
                       "l2": "flushed by a 256 MB device write before every timed step",
                       "parallelism": f"{world} independent replica(s), one batch per GPU"},
            "e2e": {"value": u_all * a.steps / (ms_e2e * 1e-3), "unit": "normals/s", "ms_per_step": ms_e2e / a.steps,
                    "h2d_bytes_per_step": 12 * total, "d2h_bytes_per_step": 12 * total},
            "roofline": {"bound": "hbm", "kernel": "whole batched pipeline (all kernels of one step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": None, "alg_bytes_per_launch": alg},
            "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu}), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(workload, seed, sample):
    """The reference pipeline restated on the host cores, on a bounded sample."""
    from oracle import oracle as O

    wl = _workloads()[workload]
    from shapeextraction_b200 import synth

    k = wl["k"] or 16
    n = min(sample, 100_000) if workload.startswith("cube") else sample
    x, y, z = wl["sample"](n, seed)
    O.pipeline_reference(x[:1000], y[:1000], z[:1000], k)  # warm the library
    t = time.perf_counter()
    u, _ = O.pipeline_reference(x, y, z, k)
    dt = time.perf_counter() - t
    return {"value": u / dt, "unit": "normals/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{x.size} points of the workload's generator ({wl['sample'].__name__}), k={k}: reference "
                      "pipeline restated on the host (bit-exact build, the reference's approximate octree search, "
                      "FP32 covariance, FP64 Jacobi), OpenMP on all cores", "seconds": dt}


def reference_cuda(workload, seed, reps=3, xyz=None):
    """The reference's own CUDA build (oracle/_ref/refdriver) on the full
    workload (the cloud `xyz` when given, else generated from `seed`)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "refdriver")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/refdriver not built"}
    from oracle import oracle as O
    from shapeextraction_b200 import synth

    wl = _workloads()[workload]

    def well_formed(x, y, z):
        a = O.build_stages(x, y, z, 63, root_compat=True)["radix"]
        b = O.build_stages(x, y, z, 63, root_compat=False)["radix"]
        return all(np.array_equal(a[key][:1], b[key][:1]) for key in ("leftChild", "prefixN", "hasLeafLeft",
                                                                         "hasLeafRight"))

    if wl.get("batched"):
        # the reference has no batched entry point: its API runs cloud after cloud
        clouds, ks = wl["gen"](seed)
        with tempfile.TemporaryDirectory() as tmp:
            lines, skipped, n_in = [], 0, 0
            for i, ((cx, cy, cz), kk) in enumerate(zip(clouds, ks)):
                if cx.size < 3 or not well_formed(cx, cy, cz):
                    skipped += 1
                    continue
                f = os.path.join(tmp, f"c{i}.bin")
                synth.to_cloud_file(f, cx, cy, cz)
                lines.append(f"{f} {int(kk)}")
                n_in += cx.size
            lst = os.path.join(tmp, "list.txt")
            with open(lst, "w") as fh:
                fh.write("\n".join(lines) + "\n")
            try:
                r = subprocess.run([exe, "batch", lst, "1", str(max(1, reps - 2))], capture_output=True, text=True,
                                   timeout=1500)
            except subprocess.TimeoutExpired:
                return {"unavailable": "reference CUDA build exceeded 1500 s on the batch"}
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("REFJSON ")]
        if r.returncode != 0 or not lines:
            return {"unavailable": f"refdriver exit {r.returncode}: {r.stderr[-300:]}"}
        d = json.loads(lines[-1][8:])
        ms = statistics.median(d["ms"])
        return {"value": d["u"] / (ms * 1e-3), "unit": "normals/s", "ms": d["ms"], "u": d["u"], "clouds": d["clouds"],
                "skipped_clouds": skipped, "points": n_in,
                "span": "cloud after cloud: host PointCloud in -> RadixTree ctor -> Octree ctor -> "
                        "estimateNormals<k> -> host normals",
                "build": "unmodified reference sources, nvcc 12.9 -O3 -DNDEBUG sm_100a (oracle/build_ref.sh)",
                "cuda_error": d.get("cuda_error")}
    x, y, z = xyz if xyz is not None else wl["gen"](seed)
    if not well_formed(x, y, z):
        return {"unavailable": "the reference's root range breaks this cloud's tree (it would read unset parents)"}
    with tempfile.TemporaryDirectory() as tmp:
        f = os.path.join(tmp, "cloud.bin")
        synth.to_cloud_file(f, x, y, z)
        try:
            r = subprocess.run([exe, "bench", f, str(wl["k"]), "1", str(reps)], capture_output=True, text=True,
                               timeout=900)
        except subprocess.TimeoutExpired:
            return {"unavailable": "reference CUDA build exceeded 900 s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("REFJSON ")]
    if r.returncode != 0 or not lines:
        return {"unavailable": f"refdriver exit {r.returncode}: {r.stderr[-300:]}"}
    d = json.loads(lines[-1][8:])
    ms = statistics.median(d["ms"])
    return {"value": d["u"] / (ms * 1e-3), "unit": "normals/s", "ms": d["ms"], "u": d["u"],
            "span": "host PointCloud in -> RadixTree ctor -> Octree ctor -> estimateNormals<k> -> host normals",
            "build": "unmodified reference sources, nvcc 12.9 -O3 -DNDEBUG sm_100a (oracle/build_ref.sh)",
            "cuda_error": d.get("cuda_error")}


def run_reference(a):
    world, rank, local = _dist()
    if rank != 0:
        return
    wl = _workloads()[a.workload]
    from oracle import oracle as O
    from shapeextraction_b200 import synth

    k_ref = wl["k"] or 16
    n = min(a.ref_sample, 100_000) if a.workload.startswith("cube") else a.ref_sample
    x, y, z = wl["sample"](n, a.seed)
    for _ in range(a.warmup):
        O.pipeline_reference(x, y, z, k_ref)
    times = []
    u = 0
    for _ in range(a.steps):
        t = time.perf_counter()
        u, _ = O.pipeline_reference(x, y, z, k_ref)
        times.append(time.perf_counter() - t)
    tot = sum(times)
    value = u * a.steps / tot
    sample = (f"{x.size} points of the workload's generator ({wl['sample'].__name__}) per step, k={k_ref}: reference "
              "pipeline restated on the host (bit-exact build, the reference's approximate octree search, FP32 "
              "covariance, FP64 Jacobi)")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "normals/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": tot / a.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": a.workload, "desc": wl["desc"], "k": k_ref, "code_bits": wl["code_bits"],
                   "sample_points_per_step": int(x.size), "unique_points_per_step": int(u)},
        "cpu_baseline": {"value": value, "unit": "normals/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "normals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not a.no_reference_cuda:
        line["reference_cuda_build"] = reference_cuda(a.workload, a.seed)
    print(json.dumps(line), flush=True)


def run_stand_in(a):
    """CPU stand-in for the launch plumbing (--stand-in): gloo ranks, each
    timing a small numpy step, the max over ranks and the JSON line exactly as
    the GPU run reports them. It measures nothing about the path; it exists so
    that the rank launch (--gpus N) and the aggregation run without a GPU."""
    world, rank, local = _dist()
    _init_dist(world, local, backend="gloo")
    rng = np.random.default_rng(a.seed + rank)
    pts = rng.random((2048, 3), dtype=np.float32)

    def step():
        d = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
        return np.argpartition(d, 16, axis=1)[:, :16]

    for _ in range(a.warmup):
        step()
    t = time.perf_counter()
    for _ in range(a.steps):
        step()
    ms = (time.perf_counter() - t) * 1e3
    import torch

    ms = _reduce([ms], "max", torch.device("cpu"))[0]
    units = _reduce([pts.shape[0]], "sum", torch.device("cpu"))[0]
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": units * a.steps / (ms * 1e-3), "unit": "normals/s",
                          "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
                          "higher_is_better": True, "scaling": "strong" if a.mode == "sharded" else "weak",
                          "stand_in": "gloo ranks on CPU timing a numpy step; launch and aggregation only",
                          "config": {"workload": "stand-in", "mode": a.mode}}), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def _free_port():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch(a, argv):
    """Run this script under torch.distributed.run with a.gpus ranks on this
    node (one per GPU), rendezvous on 127.0.0.1; returns the exit code."""
    if not a.stand_in:
        import torch

        have = torch.cuda.device_count()
        if have < a.gpus:
            print(json.dumps({"error": f"--gpus {a.gpus} asked, {have} GPU(s) visible"}), flush=True)
            return 2
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__)] + argv
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="precision_20M_k16")
    ap.add_argument("--mode", choices=["replicas", "sharded"], default="replicas",
                    help="replicas: one cloud per rank (weak scaling); sharded: one cloud, queries split over "
                         "ranks (strong scaling)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--bucket", type=int, default=96)
    ap.add_argument("--halo", type=int, default=-1,
                    help="seed halo (-1: the library's per-k default, 16 up to k=16 and 32 above)")
    ap.add_argument("--eigengap", type=float, default=None,
                    help="FP64-redo eigengap threshold (default: the workload's, else 1e-4)")
    ap.add_argument("--cpu-sample", type=int, default=2_000_000,
                    help="points of the workload's generator for the host-core baseline")
    ap.add_argument("--ref-sample", type=int, default=200_000,
                    help="points per step of --impl reference (the host-core restatement)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true")
    ap.add_argument("--no-compat", action="store_true", help="skip the reference-compatible search timing")
    ap.add_argument("--compat-steps", type=int, default=2)
    ap.add_argument("--compat-warmup", type=int, default=1)
    ap.add_argument("--no-learned", action="store_true", help="time only the plain search")
    ap.add_argument("--skip-plain", action="store_true", help="time only the learned pipeline (profiling runs)")
    ap.add_argument("--learned-keep-seed", action="store_true",
                    help="with the learned radius, still offer the Morton-window seed")
    ap.add_argument("--train-steps", type=int, default=1500)
    ap.add_argument("--autotune", action="store_true", help="pick the batch tuning with the autotuner (cached)")
    ap.add_argument("--autotune-cache", default=os.path.join(ROOT, "_build", "autotune.json"))
    ap.add_argument("--points", type=int, default=0,
                    help="resize the workload's cloud to this many points (profiling runs; 0: the configuration's)")
    ap.add_argument("--stand-in", action="store_true", help=argparse.SUPPRESS)
    argv = sys.argv[1:]
    a = ap.parse_args(argv)
    if a.warmup < 3:
        a.warmup = 3
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(a, argv)
    if a.eigengap is None:
        a.eigengap = _workloads()[a.workload].get("eigengap", 1e-4)
    if a.stand_in:
        run_stand_in(a)
    elif a.impl == "reference":
        run_reference(a)
    elif _workloads()[a.workload].get("batched"):
        run_batch(a)
    else:
        run_ours(a)
    return 0


if __name__ == "__main__":
    sys.exit(main())
