"""Precision configuration: 20M points mixing well-conditioned surfaces with
near-degenerate neighbourhoods (anisotropic-noise planes, collinear segments,
1e-4-scale clusters offset by 1e3). Normals from the GPU path are compared
with the FP64 oracle (exact kNN set, FP64 covariance and Jacobi) on a sample
of queries; angular errors are reported separately by the oracle's relative
eigengap (l1 - l0) / l2, for the FP64-redo threshold of the configuration
(1e-6) and the library default (1e-4). At the configuration's threshold the
self-query kNN path (the one that produces the normals) is checked bit-exact
on 64 Morton-contiguous slices, plain and with the learned radius. Set
SHAPEX_REPORT_DIR to keep the report as JSON."""
import json
import os

import numpy as np
import pytest

from conftest import angle_deg_free
from shapeextraction_b200 import learned, synth
from test_configs import check_knn_rows, slices

pytestmark = pytest.mark.gpu


def _stats(a):
    if a.size == 0:
        return {"count": 0}
    return {"count": int(a.size), "p50": float(np.median(a)), "p99": float(np.quantile(a, 0.99)),
            "max": float(a.max())}


def test_precision_mix_20M(native, oracle):
    n = int(os.environ.get("SHAPEX_PRECISION_N", 20_000_000))
    x, y, z = synth.precision_mix(n, seed=4)
    rng = np.random.default_rng(0)
    report = {"n_input": n}
    with native.Context(eigengap_fp64=1e-6) as c:
        info = c.build(x, y, z)
        u = info["n_points"]
        report.update({"unique_points": u, "dedup_collapse": 1.0 - u / n, "octree_nodes": info["n_octree"]})
        pts = c.points()
        q = np.sort(rng.choice(u, size=min(200_000, u), replace=False))
        ei, _ = oracle.knn_exact(pts, pts[q], 16)
        ref, ev = oracle.normals_f64(pts, ei, pts[q])
        gap = (ev[:, 1] - ev[:, 0]) / np.maximum(np.abs(ev[:, 2]), 1e-300)
        classes = {"gap>=1e-3": gap >= 1e-3, "1e-6<=gap<1e-3": (gap >= 1e-6) & (gap < 1e-3), "gap<1e-6": gap < 1e-6}
        for thr in (1e-6, 1e-4):
            with native.Context(eigengap_fp64=thr) as c2:
                c2.build(x, y, z)
                nrm = c2.normals(16)
                fp64 = c2.stats()["fp64_solves"]  # counters of the last query call
                if thr == 1e-4:
                    # external queries at the sampled points find the same lists
                    assert np.array_equal(c2.knn(pts[q], 16), ei)
                else:
                    # the configuration's own threshold, as the bench runs it:
                    # the self-query path (the rows that produce the normals)
                    # bit-exact on 64 Morton-contiguous slices, plain and with
                    # the learned radius, whose normals equal the plain ones
                    ranges = slices(u)
                    check_knn_rows(c2, oracle, pts, 16, ranges)
                    with native.Context() as t:
                        t.build(*synth.precision_mix(2_000_000, 101))
                        rep_l = learned.train_radius_model(t, 16, steps=600)
                        c2.mlp_params(t.mlp_params())
                    c2.mlp_set_margin(rep_l["margin"])
                    c2.set_learned(True, skip_seed=True)
                    check_knn_rows(c2, oracle, pts, 16, ranges)
                    assert np.array_equal(c2.normals(16), nrm)
                    report["learned_misses"] = c2.stats()["learned_misses"]
            ang = angle_deg_free(nrm[q], ref)
            rep = {"fp64_solves": fp64, "fp64_fraction": fp64 / u}
            for name, m in classes.items():
                rep[name] = _stats(ang[m])
            report[f"eigengap_fp64={thr:g}"] = rep
            # well-conditioned neighbourhoods meet the 1e-3 rad bar
            assert rep["gap>=1e-3"]["count"] > 0
            assert rep["gap>=1e-3"]["max"] <= 1e-3
    out = os.environ.get("SHAPEX_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "precision_20M.json"), "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report))
