"""Failure detection on the device, made to fire without faulting or hanging
the GPU. The reference's checks only print (src/CudaCommon.hpp:23-76); here
every bounded wait and cap ends in a status the host reads, and the context
stays usable. The test hooks of se_options (debug_wait_limit, debug_inject)
are one-shot: each fires on the next call that reaches it.

- A decoupled look-back whose predecessor never publishes (the first sort tile
  is told not to) gives up after debug_wait_limit polls: SE_ERR_SYNC_TIMEOUT,
  and the kernels return on their own.
- A kNN walk capped at one node visit per warp: SE_ERR_SEARCH_LIMIT.
- A build-buffer allocation that fails as cudaMalloc would: SE_ERR_OOM.
After each, the same context builds and queries correctly (against the CPU
oracle)."""
import time

import numpy as np
import pytest

from shapeextraction_b200 import synth

pytestmark = pytest.mark.gpu


def _check_ok(c, oracle, x, y, z):
    info = c.build(x, y, z)
    ref = oracle.build_stages(x, y, z)
    assert info["n_points"] == ref["codes"].size
    assert np.array_equal(c.codes(), ref["codes"])
    pts = c.points()
    idx = c.knn_self(8)
    ei, _ = oracle.knn_exact(pts, pts, 8)
    assert np.array_equal(idx, ei)


def test_lookback_wait_runs_out_then_context_recovers(native, oracle):
    x, y, z = synth.scene(200_000, 41)
    with native.Context(debug_wait_limit=2000, debug_inject=native.SE_DEBUG_STALL_SORT_TILE) as c:
        t0 = time.perf_counter()
        with pytest.raises(native.ShapexError) as e:
            c.build(x, y, z)
        dt = time.perf_counter() - t0
        assert e.value.status == 8, e.value  # SE_ERR_SYNC_TIMEOUT
        assert dt < 30.0  # the waits ended by themselves
        # a failed build is not a build: queries are refused
        with pytest.raises(native.ShapexError) as e:
            c.normals(8)
        assert e.value.status == 4  # SE_ERR_NOT_BUILT
        _check_ok(c, oracle, x, y, z)


def test_search_limit_then_context_recovers(native, oracle):
    x, y, z = synth.scene(100_000, 42)
    with native.Context(debug_inject=native.SE_DEBUG_SEARCH_LIMIT) as c:
        c.build(x, y, z)
        with pytest.raises(native.ShapexError) as e:
            c.normals(16)
        assert e.value.status == 6, e.value  # SE_ERR_SEARCH_LIMIT
        _check_ok(c, oracle, x, y, z)


def test_allocation_failure_then_context_recovers(native, oracle):
    x, y, z = synth.scene(50_000, 43)
    with native.Context(debug_inject=native.SE_DEBUG_ALLOC_FAIL) as c:
        with pytest.raises(native.ShapexError) as e:
            c.build(x, y, z)
        assert e.value.status == 3, e.value  # SE_ERR_OOM
        _check_ok(c, oracle, x, y, z)
