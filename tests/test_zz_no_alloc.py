"""se_sort_keys_static: the entry point that allocates nothing.

It is for callers that cannot call cudaMalloc (code inside another
framework's device-memory budget, or latency-critical loops where allocation
is banned); its scratch is a static device array inside the library. This
checks it, through the C ABI, against the existing build entry point: the
sorted unique Morton codes of se_build (se_get_codes), shuffled, must come
back from se_sort_keys_static exactly, on two calls in a row that share the
static scratch, and a size above the stated maximum must be rejected.
"""
import ctypes

import numpy as np
import pytest

from shapeextraction_b200 import synth

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_static_sort_matches_build_codes(native):
    import torch

    x, y, z = synth.scene(300_000, seed=77)
    with native.Context() as c:
        c.build(x, y, z)
        codes = c.codes()  # existing entry point: ascending unique codes
    assert codes.size > 250_000
    L = native.lib()
    stream = torch.cuda.current_stream()
    ref = torch.from_numpy(codes.view(np.int64)).cuda()
    for seed in (1, 2):  # two calls in a row share (and reuse) the static scratch
        g = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(codes.size, generator=g).cuda()
        keys_in = ref[perm].contiguous()
        keys_out = torch.full_like(keys_in, -1)
        rc = L.se_sort_keys_static(_ptr(keys_in), _ptr(keys_out), keys_in.numel(),
                                   ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, native.STATUS_NAMES.get(rc, rc)
        assert torch.equal(keys_out, ref)
    # in place, on the same array
    keys = ref.flip(0).contiguous()
    assert L.se_sort_keys_static(_ptr(keys), _ptr(keys), keys.numel(), ctypes.c_void_p(stream.cuda_stream)) == 0
    assert torch.equal(keys, ref)


def test_static_sort_rejects_oversize(native):
    import torch

    L = native.lib()
    n = (1 << 20) + 1  # SE_STATIC_SORT_MAX_KEYS + 1
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    rc = L.se_sort_keys_static(_ptr(keys), _ptr(keys), n, None)
    assert rc == 1  # SE_ERR_INVALID_ARG
