"""The C++ facade (include/shapex.hpp): compiles against the header and links
against libshapex.so on CPU; on the GPU its results equal the C ABI's."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from shapeextraction_b200 import synth


def _build_facade(tmp_path, native):
    exe = str(tmp_path / "facade_main")
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    libdir = os.path.dirname(native.LIB_PATH)
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_main.cpp"), "-L", libdir, "-lshapex",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


def test_facade_compiles_and_links(tmp_path, native):
    exe = _build_facade(tmp_path, native)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_facade_matches_c_abi(tmp_path, native, oracle):
    exe = _build_facade(tmp_path, native)
    x, y, z = synth.scene(30000, 41)
    cloud = str(tmp_path / "cloud.bin")
    synth.to_cloud_file(cloud, x, y, z)
    out = str(tmp_path / "out")
    subprocess.run([exe, cloud, out], check=True)
    u, nr, m, mn, mx = open(out + ".info").read().split()
    with native.Context() as c:
        info = c.build(x, y, z)
        assert int(u) == info["n_points"] and int(nr) == info["n_radix"] and int(m) == info["n_octree"]
        assert np.float32(float(mn)) == np.float32(info["min_coord"])
        assert np.float32(float(mx)) == np.float32(info["max_coord"])
        nrm = np.fromfile(out + ".normals", np.float32).reshape(-1, 3)
        assert np.array_equal(nrm, c.normals(16))
        knn = np.fromfile(out + ".knn", np.int32).reshape(-1, 8)
        pts = c.points()
        ei, _ = oracle.knn_exact(pts, pts[: knn.shape[0]], 8)
        assert np.array_equal(knn, ei)
    assert os.path.getsize(out + ".ply") > 0
