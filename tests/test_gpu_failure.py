"""Failure detection without a GPU fault.

Every wait of the pipelined solver kernels is bounded. A context-wide limit
of one SM clock cycle makes the first wait that is not already satisfied run
out: the kernel records the wait in its error word, drains its own copies in
flight (always with the full limit) and returns, and the solve ends with
WSB_ERR_TIMEOUT for every system in flight. The context and the matrix stay
usable: with the default limit restored, the same solve gives the same
iterations and bits as before.
"""
import numpy as np
import pytest

import wgpu_solver_backend_b200 as wsb
from wgpu_solver_backend_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.fixture()
def own_ctx():
    # A context of its own, so the lowered limit cannot reach other tests.
    c = wsb.GpuContext.create("auto", 0)
    yield c
    c.set_wait_limit(0)


@pytest.mark.parametrize("layout", [wsb.LAYOUT_CSR, wsb.LAYOUT_BSR6])
def test_wait_limit_ends_the_solve_with_timeout_and_the_context_recovers(own_ctx, layout):
    ctx = own_ctx
    s = wsb.lattice_generate(10, seed=5)
    m = wsb.Matrix.create(ctx, s["row_ptr"], s["col_idx"], s["values"], s["block_starts"], layout=layout)
    kw = dict(max_iter=5000, rel_tol=1e-6)
    x_ok, r_ok = m.solve(s["b"], **kw)
    assert r_ok["rc"] == 0
    ctx.set_wait_limit(1)
    x0 = np.full(s["n"], 7.0, np.float32)
    x_to, r_to = m.solve(s["b"], x0=x0, raise_on_error=False, **kw)
    assert r_to["rc"] == _lib.TIMEOUT, (r_to, ctx.last_error())
    assert "device wait ran out" in ctx.last_error()
    assert np.array_equal(x_to, x0)  # x is written only on success
    # A batch on the same context meets the same limit.
    bt = wsb.Batch(ctx)
    bid = bt.add(m, s["b"], **kw)
    with pytest.raises(wsb.WsbError):
        bt.solve()
    _, rb = bt.result(bid, s["n"])
    assert rb["rc"] == _lib.TIMEOUT
    del bt
    # Default limit again: the same matrix solves as before, bit for bit.
    ctx.set_wait_limit(0)
    x2, r2 = m.solve(s["b"], **kw)
    assert r2["rc"] == 0 and r2["iterations"] == r_ok["iterations"]
    assert np.array_equal(x2.view(np.uint32), x_ok.view(np.uint32))
    bt = wsb.Batch(ctx)
    bid = bt.add(m, s["b"], **kw)
    bt.solve()
    xb, rb = bt.result(bid, s["n"])
    assert rb["rc"] == 0 and rb["iterations"] == r_ok["iterations"]
    assert np.array_equal(xb.view(np.uint32), x_ok.view(np.uint32))
