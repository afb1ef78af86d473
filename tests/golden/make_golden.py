"""Generate golden vectors from the reference's own CUDA build.

Runs oracle/_ref/refdriver (the unmodified reference sources compiled by
oracle/build_ref.sh; needs an sm_100 GPU) on seeded synthetic clouds and packs
every intermediate array it dumps into tests/golden/<case>.npz:
codes, radix arrays (prefixN, leftChild, parent, hasLeafLeft/Right), octree
nodes, decoded points, the reference's kNN indices and its normals.

Before a cloud is given to the reference, the CPU oracle checks that its radix
tree is well formed under the reference's root range (src/RadixTree.cu:128-130):
on a cloud where that root orphans a node the reference reads uninitialised
parent entries, so such clouds are skipped rather than run.

    python tests/golden/make_golden.py --out tests/golden
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from shapeextraction_b200 import synth  # noqa: E402

REFDRIVER = os.path.join(ROOT, "oracle", "_ref", "refdriver")

CASES = [
    ("cube_2k_k10", lambda: synth.uniform_cube(2000, 101), 10),
    ("scene_5k_k16", lambda: synth.scene(5000, 102), 16),
    ("dups_600_k8", lambda: synth.tiny_cloud(600, 103), 8),
    ("scene_3k_k32", lambda: synth.scene(3000, 104), 32),
]
N_SMALL = 24  # small clouds (4..40 points), the compat-root region


def well_formed(x, y, z):
    a = O.build_stages(x, y, z, 63, root_compat=True)
    b = O.build_stages(x, y, z, 63, root_compat=False)
    same = all(np.array_equal(a["radix"][k][:1], b["radix"][k][:1])
               for k in ("leftChild", "prefixN", "hasLeafLeft", "hasLeafRight"))
    return same and a["codes"].size >= 3


def run_case(x, y, z, k, tmp):
    cloud = os.path.join(tmp, "cloud.bin")
    synth.to_cloud_file(cloud, x, y, z)
    out = os.path.join(tmp, "out")
    os.makedirs(out, exist_ok=True)
    r = subprocess.run([REFDRIVER, "dump", cloud, out, str(k)], capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        raise RuntimeError(f"refdriver failed: {r.stdout[-2000:]} {r.stderr[-2000:]}")
    meta = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("REFJSON ")][-1][8:])
    u, nr, m = meta["u"], meta["n_radix"], meta["n_oct"]
    rd = lambda name, dt: np.fromfile(os.path.join(out, name), dtype=dt)  # noqa: E731
    return {
        "x": x, "y": y, "z": z, "k": np.int32(k),
        "min": np.float32(meta["min"]), "max": np.float32(meta["max"]),
        "codes": rd("codes.bin", np.uint64)[:u],
        "prefixN": rd("prefixN.bin", np.uint8)[:nr],
        "leftChild": rd("leftChild.bin", np.int32)[:nr],
        "parent": rd("parent.bin", np.int32)[:u],
        "hasLeafLeft": rd("hasLeafLeft.bin", np.uint8)[:nr],
        "hasLeafRight": rd("hasLeafRight.bin", np.uint8)[:nr],
        "nodes": rd("nodes.bin", np.uint8)[: 56 * m],
        "points": rd("points.bin", np.float32)[: 3 * u].reshape(u, 3),
        "knn": rd("knn.bin", np.int32)[: u * k].reshape(u, k),
        "normals": rd("normals.bin", np.float32)[: 3 * u].reshape(u, 3),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not os.path.exists(REFDRIVER):
        sys.exit(f"{REFDRIVER} missing: build it with oracle/build_ref.sh")
    os.makedirs(a.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name, gen, k in CASES:
            x, y, z = gen()
            if not well_formed(x, y, z):
                print(f"skip {name}: compat root breaks its tree")
                continue
            d = run_case(x, y, z, k, tmp)
            np.savez_compressed(os.path.join(a.out, name + ".npz"), **d)
            print(f"wrote {name}: u={d['codes'].size} nodes={d['nodes'].size // 56}")
        small = {}
        s = 0
        i = 0
        while i < N_SMALL and s < 500:
            n = 4 + (s % 37)
            x, y, z = synth.uniform_cube(n, seed=5000 + s)
            s += 1
            if not well_formed(x, y, z):
                continue
            d = run_case(x, y, z, 8, tmp)
            for key, v in d.items():
                small[f"{i}_{key}"] = v
            i += 1
        small["count"] = np.int32(i)
        np.savez_compressed(os.path.join(a.out, "small_clouds_k8.npz"), **small)
        print(f"wrote small_clouds_k8: {i} clouds")


if __name__ == "__main__":
    main()
