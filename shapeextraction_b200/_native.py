"""ctypes binding of libshapex.so (the C ABI declared in include/shapex.h).

The product path: every call goes to the sm_100a kernels through the C ABI.
There is no CPU fallback; a missing library or a missing GPU raises.
Arrays: numpy arrays are host memory (SE_MEM_HOST); torch CUDA tensors are
device memory (SE_MEM_DEVICE) and are used in place.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libshapex.so")

SE_OK = 0
STATUS_NAMES = {
    0: "SE_OK", 1: "SE_ERR_INVALID_ARG", 2: "SE_ERR_CUDA", 3: "SE_ERR_OOM", 4: "SE_ERR_NOT_BUILT",
    5: "SE_ERR_NONFINITE", 6: "SE_ERR_SEARCH_LIMIT", 7: "SE_ERR_DEVICE_CHECK", 8: "SE_ERR_SYNC_TIMEOUT",
    9: "SE_ERR_UNSUPPORTED",
}
SE_MEM_HOST = 0
SE_MEM_DEVICE = 1
# se_options.debug_inject bits (test hooks for the failure paths)
SE_DEBUG_STALL_SORT_TILE = 1
SE_DEBUG_SEARCH_LIMIT = 2
SE_DEBUG_ALLOC_FAIL = 4

# Every entry point declared in include/shapex.h.
EXPORTS = [
    "se_options_init", "se_status_string", "se_abi_version", "se_create", "se_destroy", "se_last_error",
    "se_build", "se_get_info", "se_get_device_views", "se_get_codes", "se_get_radix", "se_get_octree",
    "se_get_points", "se_knn_self", "se_knn", "se_normals", "se_get_stats", "se_get_profile", "se_synchronize",
    "se_sort_keys_static", "se_features", "se_mlp_init", "se_mlp_params", "se_mlp_enable", "se_mlp_set_margin", "se_mlp_forward",
    "se_mlp_predict", "se_mlp_grad", "se_mlp_train", "se_mlp_save", "se_mlp_load", "se_normals_batch",
    "se_get_batch_tuning", "se_set_batch_tuning", "se_tune_batch", "se_mlp_set_loss",
]
MLP_FEATURES = 32
MLP_PARAMS = 6337

OTNODE_DTYPE = np.dtype([
    ("children", "<i4", (8,)), ("corner", "<f4", (3,)), ("cell_size", "<f4"),
    ("child_node_mask", "<i4"), ("child_leaf_mask", "<i4"),
])


class SeOptions(ctypes.Structure):
    _fields_ = [
        ("code_bits", ctypes.c_int32), ("root_compat", ctypes.c_int32), ("build_octree", ctypes.c_int32),
        ("viewpoint", ctypes.c_float * 3), ("eigengap_fp64", ctypes.c_float), ("leaf_bucket", ctypes.c_int32),
        ("device", ctypes.c_int32), ("stream", ctypes.c_void_p), ("seed_halo", ctypes.c_int32),
        ("learned", ctypes.c_int32), ("learned_skip_seed", ctypes.c_int32), ("search_compat", ctypes.c_int32),
        ("batch_graph", ctypes.c_int32), ("debug_wait_limit", ctypes.c_int32),
        ("debug_inject", ctypes.c_int32), ("learned_cell_scan", ctypes.c_int32),
        ("cell_span", ctypes.c_int32), ("cell_max_points", ctypes.c_int32),
        ("batch_lanes", ctypes.c_int32), ("batch_lane_min_points", ctypes.c_int32),
        ("batch_blocks_per_sm", ctypes.c_int32), ("batch_warps_per_block", ctypes.c_int32),
    ]


TUNING_FIELDS = ["leaf_bucket", "seed_halo", "lanes", "lane_min_points", "blocks_per_sm", "warps_per_block"]


class SeBatchTuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in TUNING_FIELDS]


class SeInfo(ctypes.Structure):
    _fields_ = [
        ("n_input", ctypes.c_int64), ("n_points", ctypes.c_int64), ("n_radix", ctypes.c_int64),
        ("n_octree", ctypes.c_int64), ("min_coord", ctypes.c_float), ("max_coord", ctypes.c_float),
        ("code_bits", ctypes.c_int32), ("root_level", ctypes.c_int32),
    ]


class SeDeviceViews(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "codes", "points", "octree", "left_child", "parent", "prefix_n", "has_leaf_left", "has_leaf_right")]


STAT_NAMES = ["fp64_solves", "nodes_visited", "buckets_scanned", "candidates", "merge_steps", "inserts",
              "learned_misses", "cell_warps", "cell_fallbacks", "cell_lookups", "cell_points"]


class SeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in STAT_NAMES]


class SeProfile(ctypes.Structure):
    _fields_ = [("build_ms", ctypes.c_float * 8), ("query_ms", ctypes.c_float),
                ("build_launches", ctypes.c_int32), ("query_launches", ctypes.c_int32)]


BUILD_STAGES = ["bbox", "encode", "sort", "dedup_decode", "radix_tree", "search_boxes", "octree", "total"]


class ShapexError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    """Load libshapex.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m shapeextraction_b200.build` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        sigs = {
            "se_options_init": (i32, [ctypes.POINTER(SeOptions)]),
            "se_status_string": (ctypes.c_char_p, [i32]),
            "se_abi_version": (i32, []),
            "se_create": (i32, [ctypes.POINTER(P), ctypes.POINTER(SeOptions)]),
            "se_destroy": (i32, [P]),
            "se_last_error": (ctypes.c_char_p, [P]),
            "se_build": (i32, [P, P, P, P, i64, i32]),
            "se_get_info": (i32, [P, ctypes.POINTER(SeInfo)]),
            "se_get_device_views": (i32, [P, ctypes.POINTER(SeDeviceViews)]),
            "se_get_codes": (i32, [P, P, i32]),
            "se_get_radix": (i32, [P, P, P, P, P, P, i32]),
            "se_get_octree": (i32, [P, P, i32]),
            "se_get_points": (i32, [P, P, i32]),
            "se_knn_self": (i32, [P, i32, i64, i64, P, P, i32]),
            "se_knn": (i32, [P, i32, P, i64, P, P, i32]),
            "se_normals": (i32, [P, i32, i64, i64, P, i32]),
            "se_get_stats": (i32, [P, ctypes.POINTER(SeStats)]),
            "se_get_profile": (i32, [P, ctypes.POINTER(SeProfile)]),
            "se_synchronize": (i32, [P]),
            "se_sort_keys_static": (i32, [P, P, i64, P]),
            "se_features": (i32, [P, i64, i64, P, i32]),
            "se_mlp_init": (i32, [P, ctypes.c_uint64]),
            "se_mlp_params": (i32, [P, P, i32, i32]),
            "se_mlp_enable": (i32, [P, i32, i32]),
            "se_mlp_set_margin": (i32, [P, ctypes.c_float]),
            "se_mlp_set_loss": (i32, [P, ctypes.c_float]),
            "se_mlp_forward": (i32, [P, P, i64, P, i32]),
            "se_mlp_predict": (i32, [P, i64, i64, P, P, i32]),
            "se_mlp_grad": (i32, [P, P, P, i64, P, P, i32]),
            "se_mlp_train": (i32, [P, P, P, i64, i32, i32, ctypes.c_float, P, i32]),
            "se_mlp_save": (i32, [P, ctypes.c_char_p]),
            "se_mlp_load": (i32, [P, ctypes.c_char_p]),
            "se_normals_batch": (i32, [P, P, P, P, P, i32, P, P, P, i32]),
            "se_get_batch_tuning": (i32, [P, ctypes.POINTER(SeBatchTuning)]),
            "se_set_batch_tuning": (i32, [P, ctypes.POINTER(SeBatchTuning)]),
            "se_tune_batch": (i32, [P, P, P, P, P, i32, P, i32, i32, ctypes.POINTER(SeBatchTuning),
                                    ctypes.POINTER(ctypes.c_float)]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _ptr(a):
    """(pointer, mem) of a numpy array (host) or torch tensor (device if CUDA)."""
    if a is None:
        return None, SE_MEM_HOST
    if _is_torch(a):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr()), (SE_MEM_DEVICE if a.is_cuda else SE_MEM_HOST)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(ctypes.c_void_p), SE_MEM_HOST


class Context:
    """One se_ctx: device memory and a CUDA stream for one host thread."""

    def __init__(self, code_bits=63, root_compat=True, build_octree=True, viewpoint=(0.0, 0.0, 0.0),
                 eigengap_fp64=1e-4, leaf_bucket=96, device=0, stream=None, seed_halo=-1, learned=False,
                 learned_skip_seed=False, search_compat=False, batch_graph=True, debug_wait_limit=0,
                 debug_inject=0, learned_cell_scan=False, cell_span=0, cell_max_points=0, batch_lanes=0,
                 batch_lane_min_points=0, batch_blocks_per_sm=0, batch_warps_per_block=0):
        L = lib()
        o = SeOptions()
        L.se_options_init(ctypes.byref(o))
        o.code_bits = code_bits
        o.root_compat = int(bool(root_compat))
        o.build_octree = int(bool(build_octree))
        for i in range(3):
            o.viewpoint[i] = float(viewpoint[i])
        o.eigengap_fp64 = float(eigengap_fp64)
        o.leaf_bucket = int(leaf_bucket)
        o.device = int(device)
        o.stream = stream
        o.seed_halo = int(seed_halo)
        o.learned = int(bool(learned))
        o.learned_skip_seed = int(bool(learned_skip_seed))
        o.search_compat = int(bool(search_compat))
        o.batch_graph = int(bool(batch_graph))
        o.debug_wait_limit = int(debug_wait_limit)
        o.debug_inject = int(debug_inject)
        o.learned_cell_scan = int(bool(learned_cell_scan))
        o.cell_span = int(cell_span)
        o.cell_max_points = int(cell_max_points)
        o.batch_lanes = int(batch_lanes)
        o.batch_lane_min_points = int(batch_lane_min_points)
        o.batch_blocks_per_sm = int(batch_blocks_per_sm)
        o.batch_warps_per_block = int(batch_warps_per_block)
        self.options = o
        h = ctypes.c_void_p()
        rc = L.se_create(ctypes.byref(h), ctypes.byref(o))
        if rc != SE_OK:
            raise ShapexError(rc, "se_create failed (no sm_100 GPU, or bad options)")
        self._h = h
        self._built = False

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().se_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != SE_OK:
            msg = lib().se_last_error(self._h)
            raise ShapexError(rc, f"{what}: {msg.decode() if msg else ''}")

    @property
    def handle(self):
        return self._h

    # -- build --------------------------------------------------------------
    def build(self, x, y, z):
        n = len(x)
        if not (len(y) == n and len(z) == n):
            raise ValueError("x, y, z lengths differ")
        if not _is_torch(x):
            x, y, z = (np.ascontiguousarray(a, dtype=np.float32) for a in (x, y, z))
        px, mem = _ptr(x)
        py, _ = _ptr(y)
        pz, _ = _ptr(z)
        self._keep = (x, y, z)
        self._check(lib().se_build(self._h, px, py, pz, n, mem), "se_build")
        self._keep = None
        self._built = True
        return self.info()

    def info(self):
        i = SeInfo()
        self._check(lib().se_get_info(self._h, ctypes.byref(i)), "se_get_info")
        return {"n_input": i.n_input, "n_points": i.n_points, "n_radix": i.n_radix, "n_octree": i.n_octree,
                "min_coord": i.min_coord, "max_coord": i.max_coord, "code_bits": i.code_bits,
                "root_level": i.root_level}

    def device_views(self):
        v = SeDeviceViews()
        self._check(lib().se_get_device_views(self._h, ctypes.byref(v)), "se_get_device_views")
        return {n: getattr(v, n) for n, _ in SeDeviceViews._fields_}

    # -- stage copies -------------------------------------------------------
    def codes(self):
        u = self.info()["n_points"]
        out = np.zeros(u, np.uint64)
        self._check(lib().se_get_codes(self._h, _ptr(out)[0], SE_MEM_HOST), "se_get_codes")
        return out

    def radix(self):
        inf = self.info()
        u, nr = inf["n_points"], inf["n_radix"]
        r = {"leftChild": np.zeros(nr, np.int32), "parent": np.zeros(max(u, 1), np.int32),
             "prefixN": np.zeros(nr, np.uint8), "hasLeafLeft": np.zeros(nr, np.uint8),
             "hasLeafRight": np.zeros(nr, np.uint8)}
        self._check(lib().se_get_radix(self._h, _ptr(r["leftChild"])[0], _ptr(r["parent"])[0], _ptr(r["prefixN"])[0],
                                       _ptr(r["hasLeafLeft"])[0], _ptr(r["hasLeafRight"])[0], SE_MEM_HOST),
                    "se_get_radix")
        return r

    def octree(self):
        m = self.info()["n_octree"]
        out = np.zeros(m, OTNODE_DTYPE)
        self._check(lib().se_get_octree(self._h, _ptr(out)[0], SE_MEM_HOST), "se_get_octree")
        return out

    def points(self):
        u = self.info()["n_points"]
        out = np.zeros((u, 3), np.float32)
        self._check(lib().se_get_points(self._h, _ptr(out)[0], SE_MEM_HOST), "se_get_points")
        return out

    # -- queries ------------------------------------------------------------
    def _range(self, start, count):
        u = self.info()["n_points"]
        if count is None:
            count = u - start
        return start, count

    def knn_self(self, k, start=0, count=None, with_d2=False, out=None, out_d2=None):
        start, count = self._range(start, count)
        idx = out if out is not None else np.zeros((count, k), np.int32)
        d2 = out_d2 if out_d2 is not None else (np.zeros((count, k), np.float32) if with_d2 else None)
        pi, mem = _ptr(idx)
        pd, _ = _ptr(d2)
        self._check(lib().se_knn_self(self._h, k, start, count, pi, pd, mem), "se_knn_self")
        return (idx, d2) if with_d2 else idx

    def knn(self, queries, k, with_d2=False):
        q = queries if _is_torch(queries) else np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 3)
        nq = q.shape[0]
        if _is_torch(q):
            import torch
            idx = torch.zeros((nq, k), dtype=torch.int32, device=q.device)
            d2 = torch.zeros((nq, k), dtype=torch.float32, device=q.device) if with_d2 else None
        else:
            idx = np.zeros((nq, k), np.int32)
            d2 = np.zeros((nq, k), np.float32) if with_d2 else None
        pq, mem = _ptr(q)
        self._check(lib().se_knn(self._h, k, pq, nq, _ptr(idx)[0], _ptr(d2)[0], mem), "se_knn")
        return (idx, d2) if with_d2 else idx

    def normals(self, k, start=0, count=None, out=None):
        start, count = self._range(start, count)
        o = out if out is not None else np.zeros((count, 3), np.float32)
        po, mem = _ptr(o)
        self._check(lib().se_normals(self._h, k, start, count, po, mem), "se_normals")
        return o

    def stats(self):
        st = SeStats()
        self._check(lib().se_get_stats(self._h, ctypes.byref(st)), "se_get_stats")
        return {n: getattr(st, n) for n in STAT_NAMES}

    # -- learned search radius ----------------------------------------------
    def set_learned(self, on, skip_seed=False):
        """Switch the learned starting bound on or off for later queries."""
        self._check(lib().se_mlp_enable(self._h, int(bool(on)), int(bool(skip_seed))), "se_mlp_enable")

    def features(self, start=0, count=None):
        start, count = self._range(start, count)
        out = np.zeros((count, MLP_FEATURES), np.float32)
        self._check(lib().se_features(self._h, start, count, _ptr(out)[0], SE_MEM_HOST), "se_features")
        return out

    def mlp_init(self, seed=0):
        self._check(lib().se_mlp_init(self._h, seed), "se_mlp_init")

    def mlp_params(self, params=None):
        if params is None:
            out = np.zeros(MLP_PARAMS, np.float32)
            self._check(lib().se_mlp_params(self._h, _ptr(out)[0], 0, SE_MEM_HOST), "se_mlp_params")
            return out
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == MLP_PARAMS
        self._check(lib().se_mlp_params(self._h, _ptr(p)[0], 1, SE_MEM_HOST), "se_mlp_params")

    def mlp_set_loss(self, quantile=0.0):
        """Training loss: 0 = squared error, q in (0, 1) = pinball loss of quantile q."""
        self._check(lib().se_mlp_set_loss(self._h, float(quantile)), "se_mlp_set_loss")

    def mlp_set_margin(self, margin):
        self._check(lib().se_mlp_set_margin(self._h, float(margin)), "se_mlp_set_margin")

    def mlp_forward(self, X):
        X = np.ascontiguousarray(X, np.float32)
        out = np.zeros(X.shape[0], np.float32)
        self._check(lib().se_mlp_forward(self._h, _ptr(X)[0], X.shape[0], _ptr(out)[0], SE_MEM_HOST), "se_mlp_forward")
        return out

    def mlp_predict(self, start=0, count=None):
        start, count = self._range(start, count)
        y = np.zeros(count, np.float32)
        r2 = np.zeros(count, np.float32)
        self._check(lib().se_mlp_predict(self._h, start, count, _ptr(y)[0], _ptr(r2)[0], SE_MEM_HOST),
                    "se_mlp_predict")
        return y, r2

    def mlp_grad(self, X, y):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(lib().se_mlp_grad(self._h, _ptr(X)[0], _ptr(y)[0], X.shape[0], _ptr(g)[0], _ptr(loss)[0],
                                      SE_MEM_HOST), "se_mlp_grad")
        return float(loss[0]), g

    def mlp_train(self, X, y, steps, batch, lr):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        losses = np.zeros(max(steps, 1), np.float32)
        self._check(lib().se_mlp_train(self._h, _ptr(X)[0], _ptr(y)[0], X.shape[0], steps, batch, float(lr),
                                       _ptr(losses)[0], SE_MEM_HOST), "se_mlp_train")
        return losses[:steps]

    def mlp_save(self, path):
        self._check(lib().se_mlp_save(self._h, str(path).encode()), "se_mlp_save")

    def mlp_load(self, path):
        self._check(lib().se_mlp_load(self._h, str(path).encode()), "se_mlp_load")

    def normals_batch(self, clouds, ks, out=None):
        """Normals of many independent clouds in one call. `clouds` is a list
        of (x, y, z) arrays, or one (x, y, z) triple of concatenated torch
        tensors together with `offsets` given as ks=(ks, offsets). Returns
        (normals, offsets, u): cloud c's u[c] normals start at row offsets[c]."""
        if isinstance(ks, tuple):
            ks, offsets = ks
            x, y, z = clouds
            offsets = np.ascontiguousarray(offsets, np.int64)
        else:
            sizes = [len(cl[0]) for cl in clouds]
            offsets = np.zeros(len(clouds) + 1, np.int64)
            offsets[1:] = np.cumsum(sizes)
            x, y, z = (np.ascontiguousarray(np.concatenate([cl[i] for cl in clouds]), np.float32) for i in range(3))
        ks = np.ascontiguousarray(ks, np.int32)
        n_clouds = ks.size
        total = int(offsets[-1])
        if out is None:
            if _is_torch(x):
                import torch
                out = torch.zeros((total, 3), dtype=torch.float32, device=x.device)
            else:
                out = np.zeros((total, 3), np.float32)
        u = np.zeros(n_clouds, np.int64)
        px, mem = _ptr(x)
        self._check(lib().se_normals_batch(self._h, px, _ptr(y)[0], _ptr(z)[0], _ptr(offsets)[0], n_clouds,
                                           _ptr(ks)[0], _ptr(out)[0], _ptr(u)[0], mem), "se_normals_batch")
        return out, offsets, u

    def batch_tuning(self):
        """The bucket, halo and batch scheduling se_normals_batch uses."""
        t = SeBatchTuning()
        self._check(lib().se_get_batch_tuning(self._h, ctypes.byref(t)), "se_get_batch_tuning")
        return {n: getattr(t, n) for n in TUNING_FIELDS}

    def set_batch_tuning(self, tuning):
        t = SeBatchTuning(**{n: int(tuning[n]) for n in TUNING_FIELDS})
        self._check(lib().se_set_batch_tuning(self._h, ctypes.byref(t)), "se_set_batch_tuning")

    def tune_batch(self, clouds, ks, reps=3):
        """se_tune_batch on this batch (the arguments of normals_batch): leaves
        the fastest tuning set on the context; returns it with its time (ms)."""
        if isinstance(ks, tuple):
            ks, offsets = ks
            x, y, z = clouds
            offsets = np.ascontiguousarray(offsets, np.int64)
        else:
            sizes = [len(cl[0]) for cl in clouds]
            offsets = np.zeros(len(clouds) + 1, np.int64)
            offsets[1:] = np.cumsum(sizes)
            x, y, z = (np.ascontiguousarray(np.concatenate([cl[i] for cl in clouds]), np.float32) for i in range(3))
        ks = np.ascontiguousarray(ks, np.int32)
        t = SeBatchTuning()
        ms = ctypes.c_float()
        px, mem = _ptr(x)
        self._check(lib().se_tune_batch(self._h, px, _ptr(y)[0], _ptr(z)[0], _ptr(offsets)[0], ks.size, _ptr(ks)[0],
                                        mem, int(reps), ctypes.byref(t), ctypes.byref(ms)), "se_tune_batch")
        return {**{n: getattr(t, n) for n in TUNING_FIELDS}, "ms": float(ms.value)}

    def profile(self):
        p = SeProfile()
        self._check(lib().se_get_profile(self._h, ctypes.byref(p)), "se_get_profile")
        return {"build_ms": dict(zip(BUILD_STAGES, list(p.build_ms))), "query_ms": p.query_ms,
                "build_launches": p.build_launches, "query_launches": p.query_launches}

    def synchronize(self):
        self._check(lib().se_synchronize(self._h), "se_synchronize")
