"""CPU checks of the C ABI library: it builds for sm_100a, loads, exports every
entry point include/shapex.h declares, and fails with a status (not a crash)
when no sm_100 device is present. No compute call is made here."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "shapex.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(se_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_entry_points():
    names = header_functions()
    for must in ("se_create", "se_build", "se_normals", "se_knn", "se_knn_self", "se_get_octree"):
        assert must in names


def test_library_exports_every_declared_symbol(native):
    L = native.lib()
    declared = header_functions()
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(native.EXPORTS) == declared


def test_library_is_sm100a_only(native):
    # the fatbin carries sm_100a code: its ELF notes name the arch
    blob = open(native.LIB_PATH, "rb").read()
    assert b"sm_100a" in blob


def test_options_defaults(native):
    L = native.lib()
    o = native.SeOptions()
    assert L.se_options_init(ctypes.byref(o)) == 0
    assert o.code_bits == 63 and o.root_compat == 1 and o.build_octree == 1
    assert tuple(o.viewpoint) == (0.0, 0.0, 0.0)
    assert o.search_compat == 0 and o.learned == 0 and o.batch_graph == 1
    assert o.leaf_bucket == 96 and o.seed_halo == -1  # 96-point buckets; halo picked per k
    assert ctypes.sizeof(o) == 104  # sizeof(se_options) in C: 23 four-byte fields, a pointer, 4 B padding
    assert L.se_abi_version() == 2
    assert L.se_status_string(5) == b"SE_ERR_NONFINITE"


def test_null_context_is_rejected(native):
    L = native.lib()
    assert L.se_build(None, None, None, None, 0, 0) == 1
    assert L.se_normals(None, 16, 0, 1, None, 0) == 1
    assert L.se_options_init(None) == 1


def test_create_without_gpu_fails_cleanly(native):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.ShapexError):
        native.Context()


def test_create_validates_options_before_the_device(native):
    """se_create rejects bad options with SE_ERR_INVALID_ARG before it touches
    a device, so the ranges are checked here too (leaf_bucket 1..128, seed
    halo up to 48)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = native.lib()

    def create(**kw):
        o = native.SeOptions()
        L.se_options_init(ctypes.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        h = ctypes.c_void_p()
        return L.se_create(ctypes.byref(h), ctypes.byref(o))

    for bad in ({"leaf_bucket": 129}, {"leaf_bucket": -1}, {"seed_halo": 49}, {"code_bits": 32},
                {"debug_wait_limit": -1}, {"debug_inject": 8}, {"learned_cell_scan": 2}, {"cell_span": 1},
                {"cell_span": 5}, {"cell_max_points": -1}, {"batch_lanes": 17}, {"batch_lane_min_points": -1},
                {"batch_blocks_per_sm": 33}, {"batch_warps_per_block": 3}):
        assert create(**bad) == 1, bad
    for ok in ({"leaf_bucket": 128}, {"leaf_bucket": 1}, {"leaf_bucket": 0}, {"seed_halo": 48},
               {"debug_wait_limit": 100}, {"debug_inject": 7}, {"learned_cell_scan": 1}, {"cell_span": 4},
               {"batch_lanes": 16}, {"batch_lane_min_points": 1000}, {"batch_blocks_per_sm": 2},
               {"batch_warps_per_block": 2}, {"batch_warps_per_block": 4}):
        assert create(**ok) == 2, ok  # valid options: fails only at the missing device (SE_ERR_CUDA)


def test_library_exports_only_the_c_abi(native):
    """Internal C++ helpers stay hidden; the exported se_ symbols are exactly
    the declared entry points."""
    import shutil
    import subprocess

    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True, check=True)
    names = [ln.split()[-1] for ln in out.stdout.splitlines() if ln.strip()]
    assert sorted(n for n in names if n.startswith("se_")) == header_functions()
    assert not [n for n in names if "shapex" in n]


def test_static_sort_source_allocates_nothing():
    """se_sort_keys_static's translation unit calls no allocating routine: its
    scratch is the file-scope static device array, addressed per call."""
    src = open(os.path.join(ROOT, "shapeextraction_b200", "csrc", "static_sort.cu")).read()
    code = re.sub(r"//[^\n]*", "", src)
    for name in ("cudaMalloc", "cudaMallocAsync", "cudaMallocManaged", "cudaMallocHost", "cudaHostAlloc",
                 "cudaFree", "malloc(", "new ", "regrow("):
        assert name not in code, name
    assert "static __device__ __align__(256)" in code
    assert code.count("cudaGetSymbolAddress") == 1
