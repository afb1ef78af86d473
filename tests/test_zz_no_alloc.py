"""se_sort_keys_static: the entry point that allocates nothing.

It is for callers that cannot call cudaMalloc (code inside another
framework's device-memory budget, or latency-critical loops where allocation
is banned); its scratch is a static device array inside the library. This
checks it, through the C ABI, against the existing build entry point: the
sorted unique Morton codes of se_build (se_get_codes), shuffled, must come
back from se_sort_keys_static exactly, on two calls in a row that share the
static scratch, and a size above the stated maximum must be rejected. It also
sorts full 64-bit keys (bit 63 set, many duplicates) against numpy's unsigned
sort, and checks that the device's free memory does not move across calls.
"""
import ctypes

import numpy as np
import pytest

from shapeextraction_b200 import synth

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _sort(L, keys_in, keys_out, stream):
    return L.se_sort_keys_static(_ptr(keys_in), _ptr(keys_out), keys_in.numel(), ctypes.c_void_p(stream.cuda_stream))


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
        rc = _sort(L, keys_in, keys_out, stream)
        assert rc == 0, native.STATUS_NAMES.get(rc, rc)
        assert torch.equal(keys_out, ref)
    # in place, on the same array
    keys = ref.flip(0).contiguous()
    assert _sort(L, keys, keys, stream) == 0
    assert torch.equal(keys, ref)


@pytest.mark.parametrize("n", [1, 4095, 4097, 1 << 20])
def test_static_sort_full_width_keys_with_duplicates(native, n):
    """Keys over the whole unsigned 64-bit range (bit 63 set on about half of
    them) with many repeats, against numpy's unsigned sort, twice in a row."""
    import torch

    L = native.lib()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(n)
    for rep in range(2):
        pool = rng.integers(0, np.iinfo(np.uint64).max, size=max(n // 8, 1), dtype=np.uint64, endpoint=True)
        pool[0] = np.uint64(1) << np.uint64(63)
        keys = pool[rng.integers(0, pool.size, size=n)]
        if n > 2:
            keys[:2] = [np.iinfo(np.uint64).max, 0]
        ref = np.sort(keys)
        keys_in = torch.from_numpy(keys.view(np.int64)).cuda()
        keys_out = torch.full_like(keys_in, 7)
        assert _sort(L, keys_in, keys_out, stream) == 0, rep
        assert np.array_equal(keys_out.cpu().numpy().view(np.uint64), ref), rep


def test_static_sort_allocates_no_device_memory(native):
    """The property the entry point exists for: after a first call, further
    calls leave the device's free memory where it was (cudaMemGetInfo sees
    every allocation, torch's caching allocator or not)."""
    import torch

    L = native.lib()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(3)
    keys = torch.from_numpy(rng.integers(-2**63, 2**63 - 1, size=1 << 20, dtype=np.int64)).cuda()
    out = torch.empty_like(keys)
    assert _sort(L, keys, out, stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _sort(L, keys, out, stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_sort_rejects_oversize(native):
    import torch

    L = native.lib()
    n = (1 << 20) + 1  # SE_STATIC_SORT_MAX_KEYS + 1
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    rc = L.se_sort_keys_static(_ptr(keys), _ptr(keys), n, None)
    assert rc == 1  # SE_ERR_INVALID_ARG
