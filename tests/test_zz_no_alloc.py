"""The allocation-free dot product against the allocating one.

wsb_dot_tree256_noalloc serves callers that cannot allocate device memory
where they need a dot product (a process whose memory budget is already
spent, or a loop that must not pay cudaMalloc's synchronisation); its
scratch is a static device array. Through the C ABI, two calls in a row must
give exactly the result of wsb_dot_scalar_executor_dot_into and of the CPU
oracle's 256-wide FP32 tree (dot_partials.wgsl + dot_reduce.wgsl order), so
the tolerance is bit equality, as for the other executor tests. The largest
case is the size limit itself, where the static scratch is full.
Collected last so that a stop-at-first-failure run has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import wgpu_solver_backend_b200 as wsb
from wgpu_solver_backend_b200 import _lib

MAX_N = 16_777_216  # WSB_NOALLOC_DOT_MAX_N

pytestmark = pytest.mark.gpu


def _dev_buffer(ctx, arr):
    return ctx.create_storage_buffer(np.ascontiguousarray(arr, np.float32))


@pytest.mark.parametrize("n", [1, 300, 65537, 1_000_003, MAX_N])
def test_noalloc_dot_matches_allocating_dot_twice(ctx, n):
    lib = _lib.load()
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n).astype(np.float32)
    b = rng.standard_normal(n).astype(np.float32)
    ba, bb = _dev_buffer(ctx, a), _dev_buffer(ctx, b)
    # Existing entry point (scratch allocated by the executor).
    ex = wsb.DotScalarExecutor.create(ctx, n, 1)
    ex.encode_dot_scalar_into(ba, bb, n, 0)
    want = ex.readback_scalar_results()[0]
    # Allocation-free entry point, twice in a row on the same stream.
    out = ctx.create_storage_buffer(np.full(2, np.nan, np.float32))
    out_ptr = wsb._lib_handle().wsb_buffer_device_ptr(out.handle)
    for k in range(2):
        rc = lib.wsb_dot_tree256_noalloc(ctx.handle, C.c_void_p(ba.device_ptr), C.c_void_p(bb.device_ptr), n,
                                         C.c_void_p(out_ptr + 4 * k))
        assert rc == 0, ctx.last_error()
    got = ctx.readback(out)
    cpu = oracle.dot_tree256(a, b)
    assert np.float32(want).view(np.uint32) == np.float32(cpu).view(np.uint32)
    assert np.float32(got[0]).view(np.uint32) == np.float32(want).view(np.uint32)
    assert np.float32(got[1]).view(np.uint32) == np.float32(want).view(np.uint32)


def test_noalloc_dot_rejects_sizes_beyond_its_static_scratch(ctx):
    lib = _lib.load()
    out = ctx.create_storage_buffer(np.zeros(1, np.float32))
    a = ctx.create_storage_buffer(np.zeros(4, np.float32))
    rc = lib.wsb_dot_tree256_noalloc(ctx.handle, C.c_void_p(a.device_ptr), C.c_void_p(a.device_ptr),
                                     MAX_N + 1, C.c_void_p(out.device_ptr))
    assert rc == _lib.BAD_INPUT
    assert "static scratch limit" in ctx.last_error()
