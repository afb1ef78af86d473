"""Point-cloud file I/O (include/shapex_io.hpp and shapeextraction_b200/io.py):
the reference's DataIO formats (KITTI .bin, .obj, Semantic3D .txt) and PLY,
ASCII and binary, read and written by both sides. CPU only."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from shapeextraction_b200 import io, synth


def _cloud(n=5000, seed=3):
    return synth.scene(n, seed)


def test_kitti_roundtrip_and_limit(tmp_path):
    x, y, z = _cloud()
    p = str(tmp_path / "c.bin")
    io.save_kitti(p, x, y, z)
    assert os.path.getsize(p) == 16 * x.size
    rec = np.fromfile(p, "<f4").reshape(-1, 4)
    assert np.all(rec[:, 3] == 255.0)
    a = io.load_file(p)
    for u, v in zip(a, (x, y, z)):
        assert np.array_equal(u, v)
    b = io.load_kitti(p, num=4 * 100 + 3)  # a partial record is dropped
    assert b[0].size == 100 and np.array_equal(b[2], z[:100])


@pytest.mark.parametrize("binary", [True, False])
def test_ply_roundtrip(tmp_path, binary):
    x, y, z = _cloud()
    nrm = np.random.default_rng(0).normal(size=(x.size, 3)).astype(np.float32)
    p = str(tmp_path / "c.ply")
    io.save_ply(p, x, y, z, nrm, binary=binary)
    (a, b, c), n2 = io.load_ply(p)
    assert np.array_equal(a, x) and np.array_equal(b, y) and np.array_equal(c, z)
    assert np.array_equal(n2, nrm)
    io.save_ply(p, x, y, z, binary=binary)
    _, n3 = io.load_ply(p)
    assert n3 is None


def test_text_formats(tmp_path):
    obj = tmp_path / "m.obj"
    obj.write_text("# comment\nv 1 2 3\nvn 0 0 1\nv 4.5 -5 6e-1\nf 1 2 3\nv bad line\n")
    x, y, z = io.load_file(str(obj))
    assert x.tolist() == [1.0, 4.5] and z.tolist() == [3.0, np.float32(0.6)]
    s3d = tmp_path / "s.txt"
    s3d.write_text("1 2 3 10 20 30 40\n4 5 6 1 2 3\n7 8\n")
    x, y, z = io.load_file(str(s3d))
    assert x.tolist() == [1.0, 4.0] and y.tolist() == [2.0, 5.0]
    with pytest.raises(ValueError):
        io.load_file(str(tmp_path / "c.xyz"))


def _io_main(tmp_path, native):
    exe = str(tmp_path / "io_main")
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    libdir = os.path.dirname(native.LIB_PATH)
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "io_main.cpp"), "-L", libdir, "-lshapex",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("fmt", ["bin", "ply", "ascii_ply", "obj", "txt"])
def test_cpp_dataio_matches_python(tmp_path, native, fmt):
    exe = _io_main(tmp_path, native)
    x, y, z = _cloud(3000, 7)
    nrm = None
    if fmt == "bin":
        src = str(tmp_path / "in.bin")
        io.save_kitti(src, x, y, z)
    elif fmt in ("ply", "ascii_ply"):
        src = str(tmp_path / "in.ply")
        nrm = np.random.default_rng(1).normal(size=(x.size, 3)).astype(np.float32)
        io.save_ply(src, x, y, z, nrm, binary=fmt == "ply")
    elif fmt == "obj":
        src = str(tmp_path / "in.obj")
        with open(src, "w") as f:
            for a, b, c in zip(x, y, z):
                f.write(f"v {float(a)!r} {float(b)!r} {float(c)!r}\n")
    else:
        src = str(tmp_path / "in.txt")
        with open(src, "w") as f:
            for a, b, c in zip(x, y, z):
                f.write(f"{float(a)!r} {float(b)!r} {float(c)!r} 7 1 2 3\n")
    out = str(tmp_path / "out")
    r = subprocess.run([exe, src, out], check=True, capture_output=True, text=True)
    n, has_n = map(int, r.stdout.split())
    assert n == x.size and has_n == (nrm is not None)
    for path in (out + ".bin",):
        a = io.load_kitti(path)
        assert all(np.array_equal(u, v) for u, v in zip(a, (x, y, z)))
    (a, b, c), n2 = io.load_ply(out + ".ply")
    assert np.array_equal(a, x) and np.array_equal(c, z)
    assert (n2 is None) == (nrm is None) and (nrm is None or np.array_equal(n2, nrm))
    # the facade's ASCII writer (saveAsPly) prints with the stream default of
    # 6 significant digits, as the reference does: lossy, hence the binary writer
    (a, b, c), _ = io.load_ply(out + ".ascii.ply")
    assert np.allclose(a, x, rtol=1e-5, atol=0) and not np.array_equal(a, x)
