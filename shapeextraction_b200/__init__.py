"""B200-native (sm_100a) normal-estimation path of Wehrdo/ShapeExtraction.

Morton encode -> onesweep sort + dedup -> Karras radix tree -> octree ->
exact kNN -> covariance -> 3x3 eigensolve -> orientation, as hand-written CUDA
kernels behind a C ABI (include/shapex.h, libshapex.so).
"""
from .api import NormalEstimation, Octree, PointCloud, RadixTree  # noqa: F401
from ._native import Context, ShapexError, lib  # noqa: F401

__all__ = ["PointCloud", "RadixTree", "Octree", "NormalEstimation", "Context", "ShapexError", "lib"]
