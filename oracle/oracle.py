"""ctypes binding of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the product package. Each function
restates one stage of the reference's normal-estimation path; oracle.cpp cites
the reference file:line per stage.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

OTNODE_DTYPE = np.dtype(
    [
        ("children", "<i4", (8,)),
        ("corner", "<f4", (3,)),
        ("cell_size", "<f4"),
        ("child_node_mask", "<i4"),
        ("child_leaf_mask", "<i4"),
    ]
)
assert OTNODE_DTYPE.itemsize == 56


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        i32 = ctypes.c_int
        f32 = ctypes.c_float
        sig = {
            "or_bbox": (None, [P, P, P, i64, P, P]),
            "or_encode": (None, [P, P, P, i64, f32, f32, i32, P]),
            "or_decode": (None, [P, i64, f32, f32, i32, P]),
            "or_sort_dedup": (i64, [P, i64, P]),
            "or_karras": (None, [P, i64, i32, i32, P, P, P, P, P]),
            "or_octree_count": (i64, [P, P, i64, P, P]),
            "or_octree_build": (i64, [P, P, P, P, P, P, i64, P, P, i64, f32, f32, i32, P]),
            "or_knn_compat": (None, [P, P, P, i64, i32, i32, P, P]),
            "or_knn_exact": (None, [P, i64, P, i64, i32, P, P]),
            "or_knn_brute": (None, [P, i64, P, i64, i32, P, P]),
            "or_normals_f64": (None, [P, P, i64, i32, P, P, P, P]),
            "or_cov_ref_f32": (None, [P, P, i64, i32, P]),
            "or_octree_check": (i32, [P, i64, P, i64, i32, i32, P]),
            "or_pipeline_reference": (i64, [P, P, P, i64, i32, P]),
            "or_mlp_grad": (i32, [P, P, P, i64, i32, ctypes.c_double, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def bbox(x, y, z):
    x, y, z = _f32(x), _f32(y), _f32(z)
    mn = np.zeros(1, np.float32)
    mx = np.zeros(1, np.float32)
    lib().or_bbox(_p(x), _p(y), _p(z), x.size, _p(mn), _p(mx))
    return float(mn[0]), float(mx[0])


def encode(x, y, z, mn, rng, code_bits=63):
    x, y, z = _f32(x), _f32(y), _f32(z)
    out = np.empty(x.size, np.uint64)
    lib().or_encode(_p(x), _p(y), _p(z), x.size, mn, rng, code_bits, _p(out))
    return out


def decode(codes, mn, rng, code_bits=63):
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    out = np.empty((codes.size, 3), np.float32)
    lib().or_decode(_p(codes), codes.size, mn, rng, code_bits, _p(out))
    return out


def sort_dedup(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    out = np.empty(codes.size, np.uint64)
    u = lib().or_sort_dedup(_p(codes), codes.size, _p(out))
    return out[:u].copy()


def karras(codes, code_bits=63, root_compat=True):
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    u = codes.size
    n = max(u - 1, 0)
    r = {
        "leftChild": np.zeros(n, np.int32),
        # parent has u entries as in the reference (src/RadixTree.cu:348); zeroed
        "parent": np.zeros(max(u, 1), np.int32),
        "prefixN": np.zeros(n, np.uint8),
        "hasLeafLeft": np.zeros(n, np.uint8),
        "hasLeafRight": np.zeros(n, np.uint8),
    }
    if n > 0:
        lib().or_karras(_p(codes), u, code_bits, int(bool(root_compat)), _p(r["leftChild"]), _p(r["parent"]),
                        _p(r["prefixN"]), _p(r["hasLeafLeft"]), _p(r["hasLeafRight"]))
    return r


def octree(codes, radix, mn, mx, code_bits=63):
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    n = radix["leftChild"].size
    counts = np.zeros(max(n, 1), np.int32)
    offsets = np.zeros(n + 1, np.int32)
    n_oct = lib().or_octree_count(_p(radix["prefixN"]), _p(radix["parent"]), n, _p(counts), _p(offsets))
    nodes = np.zeros(max(n_oct, 0), OTNODE_DTYPE)
    skipped = 0
    if n_oct > 0:
        skipped = lib().or_octree_build(_p(codes), _p(radix["prefixN"]), _p(radix["parent"]), _p(radix["leftChild"]),
                                        _p(radix["hasLeafLeft"]), _p(radix["hasLeafRight"]), n, _p(counts),
                                        _p(offsets), n_oct, mn, mx, code_bits, _p(nodes))
    return {"nodes": nodes, "counts": counts[:n], "offsets": offsets, "skipped": int(skipped)}


def octree_check(nodes, codes, code_bits, root_level):
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    seen = np.zeros(codes.size, np.int32)
    rc = lib().or_octree_check(_p(nodes), nodes.size, _p(codes), codes.size, code_bits, root_level, _p(seen))
    return rc, seen


def knn_compat(nodes, pts, queries, k, dist_variant=1, want_pops=False):
    pts = _f32(pts)
    queries = _f32(queries)
    nq = queries.shape[0]
    out = np.zeros((nq, k), np.int32)
    pops = np.zeros(nq, np.int32) if want_pops else None
    lib().or_knn_compat(_p(nodes), _p(pts), _p(queries), nq, k, dist_variant, _p(out), _p(pops))
    return (out, pops) if want_pops else out


def knn_exact(pts, queries, k, brute=False):
    pts = _f32(pts)
    queries = _f32(queries)
    nq = queries.shape[0]
    idx = np.zeros((nq, k), np.int32)
    d2 = np.zeros((nq, k), np.float32)
    fn = lib().or_knn_brute if brute else lib().or_knn_exact
    fn(_p(pts), pts.shape[0], _p(queries), nq, k, _p(idx), _p(d2))
    return idx, d2


def normals_f64(pts, nn, query_pts, viewpoint=(0.0, 0.0, 0.0)):
    pts = _f32(pts)
    nn = np.ascontiguousarray(nn, dtype=np.int32)
    query_pts = _f32(query_pts)
    nq, k = nn.shape
    vp = np.asarray(viewpoint, np.float32)
    normals = np.zeros((nq, 3), np.float64)
    evals = np.zeros((nq, 3), np.float64)
    lib().or_normals_f64(_p(pts), _p(nn), nq, k, _p(query_pts), _p(vp), _p(normals), _p(evals))
    return normals, evals


def cov_ref_f32(pts, nn):
    pts = _f32(pts)
    nn = np.ascontiguousarray(nn, dtype=np.int32)
    nq, k = nn.shape
    out = np.zeros((nq, 6), np.float32)
    lib().or_cov_ref_f32(_p(pts), _p(nn), nq, k, _p(out))
    return out


def build_stages(x, y, z, code_bits=63, root_compat=True):
    """bbox -> encode -> sort/dedup -> Karras -> octree -> decode, as
    RT::RadixTree + OT::Octree construct them."""
    mn, mx = bbox(x, y, z)
    codes = encode(x, y, z, mn, mx - mn, code_bits)
    uniq = sort_dedup(codes)
    radix = karras(uniq, code_bits, root_compat)
    octr = octree(uniq, radix, mn, mx, code_bits)
    pts = decode(uniq, mn, mx - mn, code_bits)
    return {"min": mn, "max": mx, "codes": uniq, "radix": radix, "octree": octr, "points": pts}


def pipeline_reference(x, y, z, k):
    """The reference pipeline restated on the host (all cores): returns (u, normals)."""
    x, y, z = _f32(x), _f32(y), _f32(z)
    out = np.zeros((x.size, 3), np.float32)
    u = lib().or_pipeline_reference(_p(x), _p(y), _p(z), x.size, k, _p(out))
    return int(u), out[:u]


MLP_PARAMS = 6337


def mlp_grad(params, X, y, round_bf16=True, quantile=0.0):
    """(yhat, loss, grads) of the learned-radius MLP's mean squared error.
    round_bf16: False (FP64 throughout), True (BF16 weights, inputs and
    activations with FP32 accumulation, as the GPU's forward), or 2 (that,
    plus the BF16 rounding of dh2 and dh1 that the tensor-core training step
    applies before its products). quantile > 0: the pinball loss of that
    quantile instead of the mean squared error."""
    params = _f32(params)
    X = _f32(X)
    y = _f32(y)
    n = X.shape[0]
    yhat = np.zeros(n, np.float64)
    grads = np.zeros(MLP_PARAMS, np.float64)
    loss = np.zeros(1, np.float64)
    mode = 2 if round_bf16 == 2 else int(bool(round_bf16))
    lib().or_mlp_grad(_p(params), _p(X), _p(y), n, mode, float(quantile), _p(yhat), _p(grads), _p(loss))
    return yhat, float(loss[0]), grads


def exact_normals(pts, k, viewpoint=(0.0, 0.0, 0.0)):
    """Exact kNN (ties by index) + FP64 PCA normals for every point."""
    idx, d2 = knn_exact(pts, pts, k)
    nrm, ev = normals_f64(pts, idx, pts, viewpoint)
    return idx, d2, nrm, ev
