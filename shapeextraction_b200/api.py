"""Reference-shaped host API over the C ABI.

Mirrors the classes a caller of Wehrdo/ShapeExtraction uses (paths relative to
the reference project root), with the same names, argument meaning and order
of construction:

    cloud = PointCloud(x, y, z)                       # src/PointCloud.hpp:105-122
    radix_tree = RadixTree(cloud)                     # src/RadixTree.hpp:36-60
    octree = Octree(radix_tree)                       # src/Octree.hpp:91-126
    normals = NormalEstimation.estimateNormals(octree, k=16)   # src/NormalEstimation.hpp:14-20

Differences, on purpose: errors raise ShapexError instead of printing
(src/CudaCommon.hpp:23-76); `k` is an argument instead of a template
parameter; knnSearch takes (points, k, eps) and does not swap N and eps
(src/Octree.hpp:232); a RadixTree owns the device context that the Octree and
the queries reuse, so nothing is rebuilt or copied between them.
"""
from __future__ import annotations

import numpy as np

from ._native import Context, ShapexError  # noqa: F401


class PointCloud:
    """SoA float coordinates (PointCloud<float>, src/PointCloud.hpp:105-122).

    x_vals/y_vals/z_vals may be numpy arrays (host) or torch CUDA tensors
    (device-resident input, used in place)."""

    def __init__(self, x_vals=None, y_vals=None, z_vals=None):
        self.x_vals = x_vals if x_vals is not None else np.zeros(0, np.float32)
        self.y_vals = y_vals if y_vals is not None else np.zeros(0, np.float32)
        self.z_vals = z_vals if z_vals is not None else np.zeros(0, np.float32)
        self.x_normals = self.y_normals = self.z_normals = None

    def setNormals(self, normals):  # src/PointCloud.cpp:3-14
        n = np.asarray(normals, np.float32).reshape(-1, 3)
        if n.shape[0] != len(self.x_vals):
            raise ValueError("normals and points differ in length")
        self.x_normals, self.y_normals, self.z_normals = (np.ascontiguousarray(n[:, i]) for i in range(3))

    def saveAsPly(self, filename):  # src/PointCloud.hpp:151-190 (binary little-endian PLY)
        x, y, z = (np.asarray(a, np.float32) for a in (self.x_vals, self.y_vals, self.z_vals))
        cols = [x, y, z]
        props = ["x", "y", "z"]
        if self.x_normals is not None:
            cols += [self.x_normals, self.y_normals, self.z_normals]
            props += ["nx", "ny", "nz"]
        header = "ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % len(x)
        header += "".join("property float %s\n" % p for p in props) + "end_header\n"
        with open(filename, "wb") as f:
            f.write(header.encode())
            np.stack(cols, axis=1).astype("<f4").tofile(f)
        return True


class RadixTree:
    """RT::RadixTree(const PointCloud<float>&), src/RadixTree.cu:305-382.

    Runs the whole device build (bbox, encode, sort, dedup, Karras tree and,
    unless build_octree=False, the octree) in one call."""

    def __init__(self, cloud: PointCloud, code_bits=63, root_compat=True, build_octree=True, viewpoint=(0, 0, 0),
                 eigengap_fp64=1e-4, leaf_bucket=96, device=0, context: Context | None = None):
        self.ctx = context or Context(code_bits=code_bits, root_compat=root_compat, build_octree=build_octree,
                                      viewpoint=viewpoint, eigengap_fp64=eigengap_fp64, leaf_bucket=leaf_bucket,
                                      device=device)
        info = self.ctx.build(cloud.x_vals, cloud.y_vals, cloud.z_vals)
        self.n_pts = info["n_points"]       # after dedup, src/RadixTree.cu:290
        self.n_nodes = info["n_radix"]      # src/RadixTree.cu:353
        self.min_coord = info["min_coord"]
        self.max_coord = info["max_coord"]

    @property
    def d_tree(self):
        """Device pointers of RT::Nodes (src/RadixTree.hpp:17-34)."""
        v = self.ctx.device_views()
        return {"mortonCode": v["codes"], "hasLeafLeft": v["has_leaf_left"], "hasLeafRight": v["has_leaf_right"],
                "prefixN": v["prefix_n"], "leftChild": v["left_child"], "parent": v["parent"]}


class Octree:
    """OT::Octree(const RT::RadixTree&), src/Octree.cu:213-319.

    The octree was built with the radix tree; this copies the decoded points to
    the host as the reference does (h_points, src/Octree.cu:317-318)."""

    def __init__(self, radix_tree: RadixTree):
        self.ctx = radix_tree.ctx
        info = self.ctx.info()
        self.n_pts = info["n_points"]
        self.n_nodes = info["n_octree"]
        self.h_points = self.ctx.points()
        v = self.ctx.device_views()
        self.u_points = v["points"]  # device Point* (AoS xyz)
        self.u_nodes = v["octree"]   # device OTNode*

    def knnSearch(self, points, k, eps=0.01):
        """Octree::knnSearch<k>(points, eps), src/Octree.hpp:214-242: exact kNN
        of arbitrary query points (eps is accepted and unused: the search is exact)."""
        return self.ctx.knn(points, k)

    def deviceKnnSearch(self, k, start=0, count=None, out=None):
        """Octree::deviceKnnSearch<k> over the tree's own points
        (src/Octree.hpp:199-212 as called by estimateNormals). `out` may be a
        torch CUDA int32 tensor (count, k)."""
        return self.ctx.knn_self(k, start, count, out=out)


class NormalEstimation:
    """NormalEstimation::estimateNormals<k>, src/NormalEstimation.hpp:196-335."""

    @staticmethod
    def estimateNormals(octree: Octree, k: int = 8, start_idx: int = 0, n: int | None = None, out=None):
        return octree.ctx.normals(k, start_idx, n, out=out)
