"""Point-cloud file I/O, the Python side of include/shapex_io.hpp.

The reference's DataIO (src/DataIO.cpp) reads KITTI velodyne scans (.bin:
float32 x, y, z, reflectance records), ASCII .obj vertices and Semantic3D .txt
rows, and PointCloud::saveAsPly writes ASCII PLY (src/PointCloud.hpp:151-190).
These functions read and write the same formats with numpy (one read per
file, vectorised parsing) and add binary little-endian PLY. Loaders return
(x, y, z) float32 arrays; PLY loaders also return normals when present.
"""
from __future__ import annotations

import os

import numpy as np


def load_file(path: str):
    """By extension: .bin (KITTI), .obj, .txt (Semantic3D), .ply. Returns (x, y, z)."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".bin":
        return load_kitti(path)
    if ext == ".obj":
        return load_obj(path)
    if ext == ".txt":
        return load_semantic3d(path)
    if ext == ".ply":
        return load_ply(path)[0]
    raise ValueError(f"unknown point-cloud file extension: {path}")


def load_kitti(path: str, num: int | None = None):
    """src/DataIO.cpp:33-57; `num` = most floats to read (4 per point)."""
    a = np.fromfile(path, dtype="<f4", count=-1 if num is None else int(num))
    a = a[: a.size - a.size % 4].reshape(-1, 4)
    return (np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1]), np.ascontiguousarray(a[:, 2]))


def save_kitti(path: str, x, y, z) -> None:
    """Reflectance 255 for every point, src/DataIO.cpp:59-77."""
    rec = np.empty((len(x), 4), "<f4")
    rec[:, 0], rec[:, 1], rec[:, 2], rec[:, 3] = x, y, z, 255.0
    rec.tofile(path)


def _rows(path: str, want: int, prefix: bytes | None = None) -> np.ndarray:
    """The first `want` numbers of every line (that has them) as float32."""
    out = []
    with open(path, "rb") as f:
        for line in f.read().splitlines():
            if prefix is not None:
                if not line.startswith(prefix):
                    continue
                line = line[len(prefix):]
            parts = line.split()
            if len(parts) < want:
                continue
            try:
                out.append([float(v) for v in parts[:want]])
            except ValueError:
                continue
    return np.asarray(out, np.float32).reshape(-1, want)


def load_obj(path: str):
    """Vertex lines "v x y z", src/DataIO.cpp:79-95."""
    r = _rows(path, 3, prefix=b"v ")
    return tuple(np.ascontiguousarray(r[:, i]) for i in range(3))


def load_semantic3d(path: str):
    """Rows of at least six numbers, x y z kept, src/DataIO.cpp:97-115."""
    r = _rows(path, 6)
    return tuple(np.ascontiguousarray(r[:, i]) for i in range(3))


def save_ply(path: str, x, y, z, normals=None, binary: bool = True) -> None:
    """PLY with float x, y, z (and nx, ny, nz): binary little-endian, or ASCII as saveAsPly."""
    n = len(x)
    fmt = "binary_little_endian" if binary else "ascii"
    head = f"ply\nformat {fmt} 1.0\nelement vertex {n}\nproperty float x\nproperty float y\nproperty float z\n"
    cols = [np.asarray(x, np.float32), np.asarray(y, np.float32), np.asarray(z, np.float32)]
    if normals is not None:
        nrm = np.asarray(normals, np.float32).reshape(n, 3)
        head += "property float nx\nproperty float ny\nproperty float nz\n"
        cols += [nrm[:, 0], nrm[:, 1], nrm[:, 2]]
    head += "end_header\n"
    rec = np.stack(cols, axis=1).astype("<f4")
    with open(path, "wb") as f:
        f.write(head.encode())
        if binary:
            f.write(rec.tobytes())
        else:
            for row in rec:
                f.write((" ".join(repr(float(v)) for v in row) + "\n").encode())


def load_ply(path: str):
    """((x, y, z), normals or None) from an ASCII or binary little-endian PLY
    whose vertex element has only float properties."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.find(b"end_header\n")
    if not data.startswith(b"ply") or end < 0:
        raise ValueError(f"not a PLY file: {path}")
    body = end + len(b"end_header\n")
    fmt, n, props, in_vertex = None, 0, [], False
    for line in data[:end].decode().splitlines():
        line = line.strip()
        if line.startswith("format "):
            fmt = line.split()[1]
        elif line.startswith("element "):
            in_vertex = line.startswith("element vertex ")
            if in_vertex:
                n = int(line.split()[2])
        elif in_vertex and line.startswith("property "):
            t, name = line.split()[1:3]
            if t != "float":
                raise ValueError(f"PLY vertex property of type {t} is not supported")
            props.append(name)
    if fmt == "binary_little_endian":
        rec = np.frombuffer(data, "<f4", count=n * len(props), offset=body).reshape(n, len(props))
    elif fmt == "ascii":
        rows = [r.split() for r in data[body:].splitlines() if r.strip()][:n]
        rec = np.asarray(rows, np.float32).reshape(n, len(props))
    else:
        raise ValueError(f"unsupported PLY format {fmt}")
    c = {p: i for i, p in enumerate(props)}
    xyz = tuple(np.ascontiguousarray(rec[:, c[a]], np.float32) for a in ("x", "y", "z"))
    nrm = None
    if all(a in c for a in ("nx", "ny", "nz")):
        nrm = np.ascontiguousarray(rec[:, [c["nx"], c["ny"], c["nz"]]], np.float32)
    return xyz, nrm
